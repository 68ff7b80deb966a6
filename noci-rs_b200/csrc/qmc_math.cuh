// Per-determinant and per-spawn arithmetic of the NOCI-QMC propagation, as __host__ __device__
// code (the CUDA kernels in qmc.cu call it on the device; the CPU tests compile it on the host).
//
// Restated from dy-cl/noci-rs src/stochastic:
//  * FRI stochastic rounding Phi_c               metric.rs:675-699 (fri), 579-673 (sample_populations)
//  * uniform excitation generator                state.rs:707-726 (child uniform over the other
//                                                determinants, pgen = 1/(N-1), ceil(|n|) attempts)
//  * spawn amplitude -dt (H - E_s^S S) n / pgen  state.rs:569-576
//  * diagonal change -dt (H - E_s^S S - E_s^I) n state.rs:653-667, ShiftSpec state.rs:80-162
//  * shift update                                metric.rs:729-751
//
// Random numbers: Philox4x32-10, the counter-based generator of Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3" (SC11), restated from the paper: ten rounds of
// two 32 x 32 -> 64-bit multiplications with the round multipliers 0xD2511F53 and 0xCD9E8D57
// and the Weyl key increments 0x9E3779B9 and 0xBB67AE85.  Every draw is addressed by
// (seed, cycle, index, purpose), so results do not depend on thread scheduling.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define NWQ_HD __host__ __device__ __forceinline__
#else
#define NWQ_HD inline
#include <cmath>
#endif

namespace nwq {

struct U4 {
  uint32_t x, y, z, w;
};

NWQ_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

NWQ_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c.x, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c.z, &hi1, &lo1);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Purposes of the draws (fourth counter word).
constexpr uint32_t kDrawSample = 1;  // FRI sampling of the persistent populations
constexpr uint32_t kDrawChild = 2;   // uniform child of a spawning attempt
constexpr uint32_t kDrawSpawn = 3;   // FRI rounding of a spawned amplitude
constexpr uint32_t kDrawChildBin = 4;  // bin and member of a learned-proposal attempt
constexpr uint32_t kDrawTrain = 5;   // minibatch draws of the proposal training
constexpr uint32_t kDrawHarvest = 6;  // thinning of the harvested attempts
constexpr uint32_t kDrawUpdate = 7;   // FRI of a report's accumulated change (direct overlap)

// Two uniform doubles in [0, 1) with 53 random bits each, for (seed, cycle, index, purpose).
NWQ_HD void uniform2(uint64_t seed, uint64_t cycle, uint64_t index, uint32_t purpose, double* u0, double* u1) {
  const U4 c{(uint32_t)index, (uint32_t)(index >> 32), (uint32_t)cycle,
             purpose | ((uint32_t)(cycle >> 32) << 8)};
  const U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t a = ((uint64_t)r.x << 32) | r.y, b = ((uint64_t)r.z << 32) | r.w;
  *u0 = (double)(a >> 11) * (1.0 / 9007199254740992.0);
  *u1 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
}

NWQ_HD double uniform1(uint64_t seed, uint64_t cycle, uint64_t index, uint32_t purpose) {
  double u0, u1;
  uniform2(seed, cycle, index, purpose, &u0, &u1);
  return u0;
}

// Phi_c(x) with the uniform u: x if x == 0, c <= 0 or |x| >= c; else sign(x) c with
// probability |x| / c, 0 otherwise (fri, metric.rs:675-699).
NWQ_HD double fri(double x, double c, double u) {
  if (x == 0.0 || c <= 0.0 || fabs(x) >= c) return x;
  return u < fabs(x) / c ? copysign(c, x) : 0.0;
}

// Spawning attempts for a sampled population n: max(1, ceil|n|), 0 for n == 0 (state.rs:702-704).
NWQ_HD uint64_t attempts(double n) {
  if (n == 0.0) return 0;
  const double a = ceil(fabs(n));
  return a < 1.0 ? 1 : (uint64_t)a;
}

// Uniform child lambda != gamma among ndet determinants from u in [0, 1) (state.rs:711-714).
NWQ_HD uint64_t uniform_child(uint64_t gamma, uint64_t ndet, double u) {
  uint64_t l = (uint64_t)(u * (double)(ndet - 1));
  if (l >= ndet - 1) l = ndet - 2;
  if (l >= gamma) ++l;
  return l;
}

// Shifts of the signed-walker propagators (ShiftSpec, state.rs:80-162) with E_s = E_s^S = es;
// the direct-overlap propagator shifts only the overlap (ShiftSpec::direct_overlap, state.rs:95-101).
enum Propagator : int32_t { kUnshifted = 0, kShifted = 1, kDoublyShifted = 2, kDdsU1 = 3, kDdsU2 = 4, kDirectOverlap = 5 };

NWQ_HD double overlap_shift(int prop, double es) {
  (void)prop;
  return es;  // every signed-walker propagator uses E_s^S = E_s (walkers.rs:349-353)
}

NWQ_HD double identity_shift(int prop, double es) {
  return (prop == kShifted || prop == kDoublyShifted) ? es : 0.0;
}

// Diagonal change -dt (H_gg - E^S S_gg - E^I) n_g (diagonal_population_change, state.rs:653-667).
NWQ_HD double diagonal_change(int prop, double dt, double es, double h, double s, double n) {
  return -dt * (h - overlap_shift(prop, es) * s - identity_shift(prop, es)) * n;
}

// Raw spawned amplitude -dt (H - E^S S) (n / attempts) / pgen (state.rs:569-576).
NWQ_HD double spawn_amplitude(int prop, double dt, double es, double h, double s, double n_per_attempt,
                              double pgen) {
  return -dt * (h - overlap_shift(prop, es) * s) * n_per_attempt / pgen;
}

// update_shift (metric.rs:729-751): once the 1-norm reached the target, damp towards a
// constant population.
NWQ_HD double updated_shift(double shift, double damping, double dt_eff, double nw, double nw_prev) {
  return shift - (damping / dt_eff) * log(nw / nw_prev);
}

}  // namespace nwq
