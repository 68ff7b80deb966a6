// C++ host interface of the B200 Wick engine, named after the noci-rs API it stands in for.
//
//   nociwick::WicksShared              <- WicksShared / WicksView (src/nonorthogonalwicks/storage.rs:35-150,
//                                         view.rs:20-147): owns the device intermediates and basis
//   nociwick::build_wicks_shared(...)  <- build_wicks_shared (src/noci/wicks.rs:133-279)
//   nociwick::calculate_hs_pairs_wicks_batched(...)
//                                      <- calculate_hs_pairs_wicks_batched (src/noci/hs.rs:72-130)
//
// Header-only RAII layer over include/nociwick.h; errors are thrown as nociwick::Error with the
// engine's status and message.  Link with libnociwick.so.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/nociwick.h"

namespace nociwick {

class Error : public std::runtime_error {
 public:
  Error(nw_status st, const std::string& what) : std::runtime_error(what), status(st) {}
  nw_status status;
};

struct AoData {  // the fields of noci-rs AoData the Wick path reads (src/lib.rs:52-76)
  int nao = 0;
  double enuc = 0.0;
  std::vector<double> s, h, eri;  // row-major; eri is (mu nu|lam sig)
};

struct References {  // reference determinants; occupied orbitals are the first nocc columns
  int nmo = 0, nocc_a = 0, nocc_b = 0;
  std::vector<double> c_alpha, c_beta;  // nref x nao x nmo
  int nref() const { return nmo ? (int)(c_alpha.size() / ((size_t)nmo * nmo)) : 0; }
};

class WicksShared {
 public:
  WicksShared(const AoData& ao, const References& refs, double tol, nw_convention convention = NW_CONVENTION_REFERENCE,
              int device = 0) {
    nw_system sys{ao.nao, refs.nmo, ao.enuc, ao.s.data(), ao.h.data(), ao.eri.data()};
    nw_refs r{refs.nref(), refs.nocc_a, refs.nocc_b, refs.c_alpha.data(), refs.c_beta.data()};
    nw_opts o{tol, (int32_t)convention, device};
    check(nw_ctx_create(&sys, &r, &o, &ctx_), "nw_ctx_create");
  }
  WicksShared(const WicksShared&) = delete;
  WicksShared& operator=(const WicksShared&) = delete;
  WicksShared(WicksShared&& other) noexcept : ctx_(std::exchange(other.ctx_, nullptr)) {}
  ~WicksShared() { nw_ctx_destroy(ctx_); }

  void build() { check(nw_build_intermediates(ctx_), "nw_build_intermediates"); }

  void set_basis(const std::vector<nw_det>& basis) {
    check(nw_set_basis(ctx_, basis.data(), basis.size()), "nw_set_basis");
  }

  // (H, S) per pair; pairs holds (a, b) index pairs into the resident basis.
  std::vector<std::pair<double, double>> hs_pairs(const std::vector<uint32_t>& pairs, void* stream = nullptr) {
    std::vector<std::pair<double, double>> out(pairs.size() / 2);
    static_assert(sizeof(std::pair<double, double>) == 2 * sizeof(double), "pair layout");
    check(nw_eval_hs_pairs(ctx_, pairs.data(), pairs.size() / 2, reinterpret_cast<double*>(out.data()), stream),
          "nw_eval_hs_pairs");
    return out;
  }

  // Device-buffer form (asynchronous on stream).
  void hs_pairs_device(const uint32_t* pairs_dev, uint64_t npairs, double* hs_dev, void* stream) {
    check(nw_eval_hs_pairs_device(ctx_, pairs_dev, npairs, hs_dev, stream), "nw_eval_hs_pairs_device");
  }

  // Fock tables from AO Fock matrices (update_wicks_fock, src/noci/wicks.rs:290-330).
  void update_fock(const std::vector<double>& fock_a, const std::vector<double>& fock_b) {
    check(nw_update_fock(ctx_, fock_a.data(), fock_b.data()), "nw_update_fock");
  }

  // (F, S) per pair; the SNOCI element is M = F - E0 S (calculate_m_pair_wicks, src/noci/m.rs:160-197).
  std::vector<std::pair<double, double>> fs_pairs(const std::vector<uint32_t>& pairs, void* stream = nullptr) {
    std::vector<std::pair<double, double>> out(pairs.size() / 2);
    check(nw_eval_fs_pairs(ctx_, pairs.data(), pairs.size() / 2, reinterpret_cast<double*>(out.data()), stream),
          "nw_eval_fs_pairs");
    return out;
  }

  // y += S x over the resident basis (device buffers of ndet doubles; the first call on a basis
  // builds the spin-factor tables; apply_overlap_sparse, src/noci/factorise/overlap.rs:434-498).
  void apply_overlap_device(const double* x_dev, double* y_dev, void* stream) {
    check(nw_apply_overlap_device(ctx_, x_dev, y_dev, stream), "nw_apply_overlap_device");
  }

  std::vector<int32_t> zero_counts(int nref) const {
    std::vector<int32_t> m(2 * (size_t)nref * nref);
    check(nw_pair_zero_counts(ctx_, m.data()), "nw_pair_zero_counts");
    return m;
  }

  nw_ctx* handle() const { return ctx_; }

 private:
  void check(nw_status st, const char* where) const {
    if (st != NW_OK) throw Error(st, std::string(where) + ": " + nw_status_string(st) + " " + nw_last_error(ctx_));
  }
  nw_ctx* ctx_ = nullptr;
};

inline WicksShared build_wicks_shared(const AoData& ao, const References& refs, double tol,
                                      nw_convention convention = NW_CONVENTION_REFERENCE, int device = 0) {
  WicksShared w(ao, refs, tol, convention, device);
  w.build();
  return w;
}

// Batched (H, S) for determinant pairs with the same-parent rules of noci-rs: pairs of one
// parent more than a double excitation apart give exactly (0, 0).
inline std::vector<std::pair<double, double>> calculate_hs_pairs_wicks_batched(
    WicksShared& wicks, const std::vector<std::pair<uint32_t, uint32_t>>& pairs, void* stream = nullptr) {
  std::vector<uint32_t> flat;
  flat.reserve(2 * pairs.size());
  for (const auto& p : pairs) {
    flat.push_back(p.first);
    flat.push_back(p.second);
  }
  return wicks.hs_pairs(flat, stream);
}

}  // namespace nociwick
