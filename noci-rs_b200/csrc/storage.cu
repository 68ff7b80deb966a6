// On-disk cache of the built intermediates: the contiguous slab of the Wick tensors in one raw
// file and the per-reference-pair tables in a metadata file, so a later process (or context)
// with the same system skips the build.  The counterpart of the reference's wicks.bin /
// wicks.meta cache (src/nonorthogonalwicks/storage.rs:19,164-240: a raw slab of slab_len
// scalars beside a versioned, serialised metadata object with the per-pair offsets and scalar
// metadata; a version mismatch is an error).  The layout of the slab is this engine's own
// (16-byte {X|Y, hcol} records and antisymmetrised jas tensors for pairs without zero-overlap
// orbitals, reference-ordered blocks for the others), so the files are this engine's format,
// not the reference's.
//
// Slab file: the slab bytes, then the Fock basis [pair, spin][M0, M1, cx0, cx1, xc0, xc1] kept
// by the build for nw_update_fock.
// Metadata file (little-endian): magic "NWWICKS1", version, sizeof(FastPair), sizeof(GenPair),
// geometry (nao, nmo, nref, nocc_a, nocc_b, convention, transform, naux), tol, enuc, a 64-bit
// hash of every input of the build (S, h, the two-electron integrals or Cholesky vectors, the
// reference orbitals), slab and Fock-basis byte counts, nfast, then per ordered reference pair
// its sort position, zero-overlap counts (alpha, beta), generic flag and its FastPair / GenPair
// tables with every device pointer replaced by its byte offset into the slab (~0 for null), and
// a final hash of all preceding metadata bytes.  Loading checks the magic, version, table sizes,
// geometry and input hash against the context, and every offset against the slab size.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"

namespace nw {
namespace {

constexpr char kMagic[8] = {'N', 'W', 'W', 'I', 'C', 'K', 'S', '1'};
constexpr uint32_t kVersion = 1;
constexpr size_t kChunk = 64ull << 20;  // pinned staging chunk of the file copies

// FNV-1a over 64-bit words (and the tail bytes): a fingerprint of the build inputs and of the
// metadata, not a cryptographic hash.
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
      uint64_t w;
      std::memcpy(&w, b + i, 8);
      h = (h ^ w) * 1099511628211ull;
    }
    for (; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
  template <class T>
  void put(const T& v) {
    add(&v, sizeof(T));
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

// Hash of a device array (downloaded through the pinned chunk).
cudaError_t hash_device(Fnv& h, const void* d, size_t bytes, void* stage) {
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t n = std::min(kChunk, bytes - o);
    const cudaError_t e = cudaMemcpy(stage, static_cast<const char*>(d) + o, n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    h.add(stage, n);
  }
  return cudaSuccess;
}

// Fingerprint of everything the build reads: geometry, thresholds and the device copies of the
// inputs.
nw_status input_hash(nw_ctx* ctx, void* stage, uint64_t* out) {
  Fnv h;
  const int geo[8] = {ctx->nao, ctx->nmo, ctx->nref, ctx->nocc_a, ctx->nocc_b, ctx->convention, ctx->transform,
                      ctx->naux};
  h.add(geo, sizeof(geo));
  h.put(ctx->tol);
  h.put(ctx->enuc);
  const size_t n2 = (size_t)ctx->nao * ctx->nao;
  const size_t cb = (size_t)ctx->nref * ctx->nao * ctx->nmo * sizeof(double);
  struct {
    const void* p;
    size_t bytes;
  } in[] = {{ctx->d_s, n2 * sizeof(double)},
            {ctx->d_h, n2 * sizeof(double)},
            {ctx->d_eri, ctx->d_eri ? n2 * n2 * sizeof(double) : 0},
            {ctx->d_chol, ctx->d_chol ? (size_t)ctx->naux * n2 * sizeof(double) : 0},
            {ctx->d_ca, cb},
            {ctx->d_cb, cb}};
  for (const auto& x : in)
    if (x.p && x.bytes) NW_CUDA(ctx, hash_device(h, x.p, x.bytes, stage));
  *out = h.h;
  return NW_OK;
}

// Device pointer <-> byte offset into the slab (~0 for null).
template <class T>
void to_offset(const T*& p, const double* base) {
  const uint64_t v = p ? (uint64_t)(reinterpret_cast<const char*>(p) - reinterpret_cast<const char*>(base)) : ~0ull;
  std::memcpy(&p, &v, sizeof(v));
}
template <class T>
bool from_offset(const T*& p, const double* base, size_t bytes) {
  uint64_t v;
  std::memcpy(&v, &p, sizeof(v));
  if (v == ~0ull) {
    p = nullptr;
    return true;
  }
  if (v >= bytes || (v & 7) != 0) return false;
  p = reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + v);
  return true;
}

// Applies f to every device-pointer field of the pair tables.
template <class F>
bool visit(FastPair& fp, F f) {
  bool ok = true;
  for (FastSpin* s : {&fp.a, &fp.b}) ok = f(s->recx) && f(s->recy) && f(s->jas) && ok;
  return f(fp.ii0) && ok;
}
template <class F>
bool visit(GenPair& gp, F f) {
  bool ok = true;
  for (GenSpin* s : {&gp.a, &gp.b}) {
    for (int i = 0; i < 2; ++i) ok = f(s->x[i]) && f(s->y[i]) && ok;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        ok = f(s->fh_t[i][j]) && ok;
        for (int k = 0; k < 2; ++k) ok = f(s->v_t[i][j][k]) && ok;
      }
    for (int i = 0; i < 10; ++i) ok = f(s->j[i]) && ok;
  }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) ok = f(gp.vab_t[i][j][k]) && f(gp.vba_t[i][j][k]) && ok;
  for (int i = 0; i < 16; ++i) ok = f(gp.ii[i >> 3][(i >> 2) & 1][(i >> 1) & 1][i & 1]) && ok;
  return ok;
}

struct Header {
  char magic[8];
  uint32_t version, fast_size, gen_size, pad0;
  int32_t geo[8];  // nao, nmo, nref, nocc_a, nocc_b, convention, transform, naux
  double tol, enuc;
  uint64_t input_hash, slab_bytes, fbase_bytes;
  int32_t nfast, pad1;
};

}  // namespace

nw_status save_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path) {
  if (!ctx->built || !ctx->d_slab || !ctx->d_fbase) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (ctx->partial) return fail(ctx, NW_ERR_STATE, "the intermediates hold one block of a blocked evaluation");
  const int npair = ctx->nref * ctx->nref;
  const size_t n2 = (size_t)ctx->nmo * ctx->nmo;
  const size_t fbase_bytes = sizeof(double) * 2 * (size_t)npair * 6 * n2;
  Pinned stage;
  if (cudaMallocHost(&stage.p, kChunk) != cudaSuccess) return fail(ctx, NW_ERR_ALLOC, "pinned staging buffer");
  Header hd{};
  std::memcpy(hd.magic, kMagic, 8);
  hd.version = kVersion;
  hd.fast_size = sizeof(FastPair);
  hd.gen_size = sizeof(GenPair);
  const int geo[8] = {ctx->nao, ctx->nmo, ctx->nref, ctx->nocc_a, ctx->nocc_b, ctx->convention, ctx->transform,
                      ctx->naux};
  std::memcpy(hd.geo, geo, sizeof(geo));
  hd.tol = ctx->tol;
  hd.enuc = ctx->enuc;
  nw_status st = input_hash(ctx, stage.p, &hd.input_hash);
  if (st != NW_OK) return st;
  hd.slab_bytes = ctx->slab_bytes;
  hd.fbase_bytes = fbase_bytes;
  hd.nfast = ctx->nfast;

  File fs;
  fs.f = std::fopen(slab_path, "wb");
  if (!fs.f) return fail(ctx, NW_ERR_IO, std::string("cannot create ") + slab_path);
  for (const auto& part : {std::make_pair((const char*)ctx->d_slab, ctx->slab_bytes),
                           std::make_pair((const char*)ctx->d_fbase, fbase_bytes)})
    for (size_t o = 0; o < part.second; o += kChunk) {
      const size_t n = std::min(kChunk, part.second - o);
      NW_CUDA(ctx, cudaMemcpy(stage.p, part.first + o, n, cudaMemcpyDeviceToHost));
      if (std::fwrite(stage.p, 1, n, fs.f) != n) return fail(ctx, NW_ERR_IO, std::string("write failed: ") + slab_path);
    }
  if (std::fclose(fs.f) != 0) {
    fs.f = nullptr;
    return fail(ctx, NW_ERR_IO, std::string("write failed: ") + slab_path);
  }
  fs.f = nullptr;

  std::vector<FastPair> fast = ctx->fast_host;
  std::vector<GenPair> gen = ctx->gen_host;
  const double* base = ctx->d_slab;
  for (int p = 0; p < npair; ++p) {
    visit(fast[p], [&](auto& ptr) {
      to_offset(ptr, base);
      return true;
    });
    visit(gen[p], [&](auto& ptr) {
      to_offset(ptr, base);
      return true;
    });
  }
  std::vector<char> meta;
  auto app = [&](const void* p, size_t n) {
    meta.insert(meta.end(), static_cast<const char*>(p), static_cast<const char*>(p) + n);
  };
  app(&hd, sizeof(hd));
  app(ctx->order_host.data(), sizeof(int32_t) * npair);
  app(ctx->m_counts.data(), sizeof(int32_t) * 2 * npair);
  app(ctx->generic_host.data(), npair);
  app(fast.data(), sizeof(FastPair) * npair);
  app(gen.data(), sizeof(GenPair) * npair);
  Fnv mh;
  mh.add(meta.data(), meta.size());
  app(&mh.h, sizeof(mh.h));
  File fm;
  fm.f = std::fopen(meta_path, "wb");
  if (!fm.f) return fail(ctx, NW_ERR_IO, std::string("cannot create ") + meta_path);
  if (std::fwrite(meta.data(), 1, meta.size(), fm.f) != meta.size() || std::fclose(fm.f) != 0) {
    fm.f = nullptr;
    return fail(ctx, NW_ERR_IO, std::string("write failed: ") + meta_path);
  }
  fm.f = nullptr;
  return NW_OK;
}

nw_status load_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path) {
  const int npair = ctx->nref * ctx->nref;
  const size_t n2 = (size_t)ctx->nmo * ctx->nmo;
  // metadata
  std::vector<char> meta;
  {
    File fm;
    fm.f = std::fopen(meta_path, "rb");
    if (!fm.f) return fail(ctx, NW_ERR_IO, std::string("cannot open ") + meta_path);
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), fm.f)) > 0) meta.insert(meta.end(), buf, buf + n);
  }
  const size_t want = sizeof(Header) + sizeof(int32_t) * 3 * npair + npair + sizeof(FastPair) * npair +
                      sizeof(GenPair) * npair + sizeof(uint64_t);
  Header hd;
  if (meta.size() < sizeof(Header)) return fail(ctx, NW_ERR_INVALID, "Wick cache metadata truncated");
  std::memcpy(&hd, meta.data(), sizeof(hd));
  if (std::memcmp(hd.magic, kMagic, 8) != 0) return fail(ctx, NW_ERR_INVALID, "not a Wick cache metadata file");
  if (hd.version != kVersion)
    return fail(ctx, NW_ERR_INVALID, "Wick cache version " + std::to_string(hd.version) +
                                         " is incompatible with expected version " + std::to_string(kVersion));
  if (hd.fast_size != sizeof(FastPair) || hd.gen_size != sizeof(GenPair))
    return fail(ctx, NW_ERR_INVALID, "Wick cache table layout differs from this build");
  if (meta.size() != want) return fail(ctx, NW_ERR_INVALID, "Wick cache metadata has the wrong size for this system");
  {
    Fnv mh;
    mh.add(meta.data(), want - sizeof(uint64_t));
    uint64_t stored;
    std::memcpy(&stored, meta.data() + want - sizeof(uint64_t), sizeof(stored));
    if (stored != mh.h) return fail(ctx, NW_ERR_INVALID, "Wick cache metadata is corrupt (hash mismatch)");
  }
  const int geo[8] = {ctx->nao, ctx->nmo, ctx->nref, ctx->nocc_a, ctx->nocc_b, ctx->convention, ctx->transform,
                      ctx->naux};
  if (std::memcmp(hd.geo, geo, sizeof(geo)) != 0 || hd.tol != ctx->tol || hd.enuc != ctx->enuc)
    return fail(ctx, NW_ERR_INVALID, "Wick cache was built for another system or other options");
  const size_t fbase_bytes = sizeof(double) * 2 * (size_t)npair * 6 * n2;
  if (hd.fbase_bytes != fbase_bytes || hd.nfast < 0 || hd.nfast > npair)
    return fail(ctx, NW_ERR_INVALID, "Wick cache metadata inconsistent with this system");
  Pinned stage;
  if (cudaMallocHost(&stage.p, kChunk) != cudaSuccess) return fail(ctx, NW_ERR_ALLOC, "pinned staging buffer");
  uint64_t ih = 0;
  nw_status st = input_hash(ctx, stage.p, &ih);
  if (st != NW_OK) return st;
  if (ih != hd.input_hash) return fail(ctx, NW_ERR_INVALID, "Wick cache was built from other integrals or orbitals");

  // tables, relocated onto the new slab below
  const char* q = meta.data() + sizeof(Header);
  std::vector<int32_t> order(npair), mcount(2 * npair);
  std::vector<char> generic(npair);
  std::vector<FastPair> fast(npair);
  std::vector<GenPair> gen(npair);
  std::memcpy(order.data(), q, sizeof(int32_t) * npair);
  q += sizeof(int32_t) * npair;
  std::memcpy(mcount.data(), q, sizeof(int32_t) * 2 * npair);
  q += sizeof(int32_t) * 2 * npair;
  std::memcpy(generic.data(), q, npair);
  q += npair;
  std::memcpy(fast.data(), q, sizeof(FastPair) * npair);
  q += sizeof(FastPair) * npair;
  std::memcpy(gen.data(), q, sizeof(GenPair) * npair);

  // slab and Fock basis
  File fs;
  fs.f = std::fopen(slab_path, "rb");
  if (!fs.f) return fail(ctx, NW_ERR_IO, std::string("cannot open ") + slab_path);
  if (std::fseek(fs.f, 0, SEEK_END) != 0) return fail(ctx, NW_ERR_IO, std::string("cannot read ") + slab_path);
  const long long fsize = std::ftell(fs.f);
  std::rewind(fs.f);
  if (fsize < 0 || (unsigned long long)fsize != hd.slab_bytes + hd.fbase_bytes)
    return fail(ctx, NW_ERR_INVALID, "Wick cache slab file has the wrong size");
  ctx->built = false;
  ctx->fock_ready = false;
  if (ctx->d_slab) cudaFree(ctx->d_slab);
  ctx->d_slab = nullptr;
  ctx->slab_bytes = 0;
  ctx->slab_capacity = 0;
  if (ctx->d_fbase) cudaFree(ctx->d_fbase);
  ctx->d_fbase = nullptr;
  if (cudaMalloc(&ctx->d_slab, std::max<size_t>(hd.slab_bytes, 256)) != cudaSuccess) {
    ctx->d_slab = nullptr;
    return fail(ctx, NW_ERR_ALLOC, "intermediate slab allocation failed");
  }
  ctx->slab_capacity = std::max<size_t>(hd.slab_bytes, 256);
  if (cudaMalloc(&ctx->d_fbase, fbase_bytes) != cudaSuccess) {
    ctx->d_fbase = nullptr;
    return fail(ctx, NW_ERR_ALLOC, "Fock basis allocation failed");
  }
  for (const auto& part : {std::make_pair((char*)ctx->d_slab, (size_t)hd.slab_bytes),
                           std::make_pair((char*)ctx->d_fbase, fbase_bytes)})
    for (size_t o = 0; o < part.second; o += kChunk) {
      const size_t n = std::min(kChunk, part.second - o);
      if (std::fread(stage.p, 1, n, fs.f) != n) return fail(ctx, NW_ERR_IO, std::string("read failed: ") + slab_path);
      NW_CUDA(ctx, cudaMemcpy(part.first + o, stage.p, n, cudaMemcpyHostToDevice));
    }
  const double* base = ctx->d_slab;
  for (int p = 0; p < npair; ++p) {
    const auto rel = [&](auto& ptr) { return from_offset(ptr, base, hd.slab_bytes); };
    if (!visit(fast[p], rel) || !visit(gen[p], rel))
      return fail(ctx, NW_ERR_INVALID, "Wick cache table offset outside the slab");
    if (order[p] < 0 || order[p] >= npair || mcount[2 * p] < 0 || mcount[2 * p + 1] < 0)
      return fail(ctx, NW_ERR_INVALID, "Wick cache metadata inconsistent with this system");
  }
  if (!ctx->d_fast) NW_CUDA(ctx, cudaMalloc(&ctx->d_fast, sizeof(FastPair) * npair));
  if (!ctx->d_gen) NW_CUDA(ctx, cudaMalloc(&ctx->d_gen, sizeof(GenPair) * npair));
  if (!ctx->d_order) NW_CUDA(ctx, cudaMalloc(&ctx->d_order, sizeof(int32_t) * npair));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_fast, fast.data(), sizeof(FastPair) * npair, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_gen, gen.data(), sizeof(GenPair) * npair, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_order, order.data(), sizeof(int32_t) * npair, cudaMemcpyHostToDevice));
  ctx->slab_bytes = hd.slab_bytes;
  ctx->nfast = hd.nfast;
  ctx->nresident = npair;
  ctx->partial = false;
  ctx->order_host = order;
  ctx->m_counts = mcount;
  ctx->generic_host = generic;
  ctx->fast_host = fast;
  ctx->gen_host = gen;
  ctx->built = true;
  return NW_OK;
}

}  // namespace nw

extern "C" {

nw_status nw_save_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path) {
  if (!ctx || !slab_path || !meta_path) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::save_intermediates(ctx, slab_path, meta_path);
}

nw_status nw_load_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path) {
  if (!ctx || !slab_path || !meta_path) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (ctx->live_qmc > 0)
    return nw::fail(ctx, NW_ERR_STATE, "a QMC object uses the intermediates (nw_qmc_destroy it first)");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::load_intermediates(ctx, slab_path, meta_path);
}

}  // extern "C"
