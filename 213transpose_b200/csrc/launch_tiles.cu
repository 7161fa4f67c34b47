// Launchers of the square-block tile swaps and of the band transposes.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "internal.h"
#include "k_tiles.cuh"

namespace t213 {

namespace {

template <typename Kern>
int64_t resident_grid(Kern kern, int threads, size_t smem, int64_t units) {
  const DevInfo &d = dev_info();
  int per_sm = 1;
  occupancy_cached((const void *)kern, threads, (int64_t)smem, 1, &per_sm);
  return std::max<int64_t>(1, std::min<int64_t>((int64_t)per_sm * d.sms, units));
}

constexpr int64_t kBandSmemCap = 200 * 1024;

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); null when the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tile-swap kernel choice.  Measured on B200 over (8192, 6144, d3) blocks of
// t = 2048: the TMA kernel with 64 x 64 tiles moves 4-byte elements at 5.98
// TB/s against 4.70 TB/s for the register kernel (32 x 32 tiles, 128-byte
// rows), while for 8- and 16-byte elements the register kernel's 32 x 32
// tiles already have 256- and 512-byte rows and it is the faster one (5.89
// and 6.05 TB/s against 5.39 and 4.89 TB/s).  So by default the TMA kernel
// takes 4-byte elements whose block side is a multiple of 64.
// T213_TILE_SWAP=tma|vec forces a kernel; T213_TILE_STAGES (ring depth),
// T213_TILE_WARPS (consumer warps), T213_TILE_TS (tile side) and
// T213_TILE_GROUP (super-tile order) set the TMA kernel's launch shape.
const char *tile_swap_choice() {
  const Variant &pv = current_variant();
  if (pv.tile == 1) return "tma";
  if (pv.tile == 2) return "vec";
  const char *v = std::getenv("T213_TILE_SWAP");
  return v ? v : "auto";
}

int env_int(const char *name, int dflt) {
  const char *v = std::getenv(name);
  const int x = v ? std::atoi(v) : 0;
  return x > 0 ? x : dflt;
}

// Tile side of the TMA kernel for an element size (elements; one tile row is
// whole 128-byte boxes and a multiple of eight 16-byte chunks).
// The preferred side (256-byte tile rows and wider read DRAM pages more
// fully) falls back to smaller sides the block side t allows.
int tma_tile_side(int eb, int64_t t) {
  static const int sides4[] = {64, 32}, sides8[] = {64, 32, 16}, sides16[] = {32, 16, 8};
  const int *sides = eb == 4 ? sides4 : eb == 8 ? sides8 : sides16;
  const int nsides = eb == 4 ? 2 : 3;
  const int want = env_int("T213_TILE_TS", eb == 4 ? 64 : eb == 8 ? 64 : 32);
  for (int i = 0; i < nsides; i++)
    if (sides[i] <= want && t % sides[i] == 0) return sides[i];
  return 0;
}

// Super-tile group of the pair order: the largest of 8, 4, 2, 1 (at most
// T213_TILE_GROUP) that divides the tile-grid side.
uint32_t tile_group(int64_t nt) {
  const int want = env_int("T213_TILE_GROUP", 4);
  for (int g = 8; g > 1; g /= 2)
    if (g <= want && nt % g == 0) return (uint32_t)g;
  return 1;
}

// Tile swap through TMA: one 3-D tensor map over the slices viewed as
// m x (n * eb) byte matrices, 128-byte boxes of TS rows.
template <int EB, int TS>
int launch_tile_swap_tma(char *data, int64_t d3, int64_t m, int64_t n, int64_t t, cudaStream_t st, LaunchStats *ls,
                         bool *launched) {
  using TT = TileTma<EB, TS>;
  *launched = false;
  auto enc = tensor_map_encoder();
  if (!enc) return T213_OK;
  const int64_t Bm = m / t, Bn = n / t, nt = t / TS;
  const int64_t pairs = nt * (nt + 1) / 2;
  const int64_t units = d3 * Bm * Bn * pairs;
  CUtensorMap tmap;
  std::memset(&tmap, 0, sizeof tmap);
  const cuuint64_t gdim[3] = {(cuuint64_t)(n * EB), (cuuint64_t)m, (cuuint64_t)d3};
  const cuuint64_t gstride[2] = {(cuuint64_t)(n * EB), (cuuint64_t)(m * n * EB)};
  const cuuint32_t box[3] = {128u, (cuuint32_t)TS, 1u};
  const cuuint32_t estride[3] = {1u, 1u, 1u};
  CUresult r = enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, data, gdim, gstride, box, estride,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return T213_OK;  // shape the encoder rejects: the caller uses the vector kernel
  const int pair_bytes = 2 * TT::TILE_BYTES;
  const int max_ns = std::max(2, (200 * 1024) / pair_bytes);
  const int ns = std::max(2, std::min(env_int("T213_TILE_STAGES", std::max(2, (128 * 1024) / pair_bytes)), max_ns));
  const int ncw = std::max(1, std::min(env_int("T213_TILE_WARPS", 16), 31));
  const int threads = 32 * (ncw + 1);
  const int64_t smem = 1024 /* alignment slack */ + 16 * (int64_t)ns + (int64_t)ns * pair_bytes;
  int rc = T213_OK;
  int *stw = device_status_word(&rc);
  if (!stw) return rc;
  auto kern = k_tile_swap_tma<EB, TS>;
  if (!kernel_attr_once((const void *)kern, smem, 1))
    return cuda_status(cudaGetLastError(), "cudaFuncSetAttribute(tile swap tma)");
  const int64_t grid = resident_grid(kern, threads, (size_t)smem, units);
  kern<<<(unsigned)grid, threads, (size_t)smem, st>>>(
      tmap, data, n, m * n, (uint32_t)units, t, FastDiv<uint32_t>((uint64_t)(Bm * Bn * pairs)),
      FastDiv<uint32_t>((uint64_t)pairs), FastDiv<uint32_t>((uint64_t)Bn), (uint32_t)nt, tile_group(nt), ns, stw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "k_tile_swap_tma launch");
  if (ls) ls->launches++;
  *launched = true;
  return T213_OK;
}

}  // namespace

// Planning target for a band: 64 KB, so three bands stay in flight per CTA.
int64_t band_smem_limit() { return 64 * 1024; }

int64_t band_smem_bytes(int64_t R, int64_t C, int eb) { return R * C * eb; }

// Largest band a launch accepts: 100 KB for the TMA-fed kernel (two buffers),
// 200 KB with padding for the fallback kernel.
bool band_fits(int64_t R, int64_t C, int eb) {
  const int64_t S = (C % 2 == 0) ? C + 1 : C;
  return R * C * eb <= kBandSmemCap / 2 || R * S * eb <= kBandSmemCap;
}

int launch_tile_swap(char *data, int64_t d3, int64_t m, int64_t n, int64_t t, int eb, cudaStream_t st,
                     LaunchStats *ls) {
  if (t <= 0 || m % t || n % t) {
    set_error("block size must divide both matrix sides");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (d3 <= 0 || m <= 0 || n <= 0) return T213_OK;
  const int64_t Bm = m / t, Bn = n / t;
  // TMA kernel: 16-byte aligned rows, a tile side that divides t, and
  // coordinates that fit the copy's 32-bit fields
  const char *choice = tile_swap_choice();
  const bool forced_tma = std::strcmp(choice, "tma") == 0;
  const int tma_ts = (eb == 4 || eb == 8 || eb == 16) ? tma_tile_side(eb, t) : 0;
  const bool tma_ok = tma_ts > 0 && (forced_tma || (std::strcmp(choice, "vec") != 0 && eb == 4 && tma_ts == 64)) && (((uintptr_t)data | (uint64_t)(n * eb)) % 16 == 0) &&
                      n * eb < (1ll << 31) && m < (1ll << 31) && d3 < (1ll << 31) &&
                      (double)d3 * Bm * Bn * ((t / tma_ts) * (t / tma_ts + 1) / 2) < 2.0e9;
  if (tma_ok) {
    bool launched = false;
    int rc = T213_OK;
    if (eb == 4)
      rc = tma_ts == 64 ? launch_tile_swap_tma<4, 64>(data, d3, m, n, t, st, ls, &launched)
                        : launch_tile_swap_tma<4, 32>(data, d3, m, n, t, st, ls, &launched);
    else if (eb == 8)
      rc = tma_ts == 64   ? launch_tile_swap_tma<8, 64>(data, d3, m, n, t, st, ls, &launched)
           : tma_ts == 32 ? launch_tile_swap_tma<8, 32>(data, d3, m, n, t, st, ls, &launched)
                          : launch_tile_swap_tma<8, 16>(data, d3, m, n, t, st, ls, &launched);
    else
      rc = tma_ts == 32   ? launch_tile_swap_tma<16, 32>(data, d3, m, n, t, st, ls, &launched)
           : tma_ts == 16 ? launch_tile_swap_tma<16, 16>(data, d3, m, n, t, st, ls, &launched)
                          : launch_tile_swap_tma<16, 8>(data, d3, m, n, t, st, ls, &launched);
    if (rc != T213_OK || launched) return rc;
  }
  const bool vec_ok = (eb >= 4) && (t % 32 == 0) && (((uintptr_t)data | (uint64_t)(n * eb)) % 16 == 0) &&
                      (double)d3 * Bm * Bn * ((t / 32) * (t / 32 + 1) / 2) < 2.0e9;
  if (vec_ok) {
    auto gov = [&](auto EBc) -> int {
      constexpr int EB = decltype(EBc)::value;
      const int64_t nt = t / 32;
      const int64_t pairs = nt * (nt + 1) / 2;
      const int64_t units = d3 * Bm * Bn * pairs;
      auto kern = k_tile_swap_vec<EB>;
      const int64_t grid = resident_grid(kern, kTileThreads, 0, units);
      kern<<<(unsigned)grid, kTileThreads, 0, st>>>(data, n, m * n, (uint32_t)units, t,
                                                    FastDiv<uint32_t>((uint64_t)(Bm * Bn * pairs)),
                                                    FastDiv<uint32_t>((uint64_t)pairs), FastDiv<uint32_t>((uint64_t)Bn),
                                                    (uint32_t)nt);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_status(e, "k_tile_swap_vec launch");
      if (ls) ls->launches++;
      return T213_OK;
    };
    if (eb == 4) return gov(IC<4>{});
    if (eb == 8) return gov(IC<8>{});
    return gov(IC<16>{});
  }
  auto go = [&](auto EBc, auto TSc) -> int {
    constexpr int EB = decltype(EBc)::value;
    constexpr int TS = decltype(TSc)::value;
    const int64_t nt = (t + TS - 1) / TS;
    const int64_t units = d3 * Bm * Bn * (nt * (nt + 1) / 2);
    auto kern = k_tile_swap<EB, TS>;
    const int64_t grid = resident_grid(kern, kTileThreads, 0, units);
    kern<<<(unsigned)grid, kTileThreads, 0, st>>>(data, n, m * n, d3, t, Bm, Bn, nt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "k_tile_swap launch");
    if (ls) ls->launches++;
    return T213_OK;
  };
  switch (eb) {
    case 1:
      return go(IC<1>{}, IC<64>{});
    case 2:
      return go(IC<2>{}, IC<64>{});
    case 4:
      return go(IC<4>{}, IC<32>{});
    case 8:
      return go(IC<8>{}, IC<32>{});
    case 16:
      return go(IC<16>{}, IC<16>{});
  }
  set_error("unsupported element size");
  return T213_ERR_UNSUPPORTED;
}

int launch_band_transpose(char *data, int64_t n_bands, int64_t R, int64_t C, int eb, cudaStream_t st,
                          LaunchStats *ls) {
  if (n_bands <= 0 || R <= 0 || C <= 0) return T213_OK;
  const int64_t smem = R * ((C % 2 == 0) ? C + 1 : C) * eb;
  if (!band_fits(R, C, eb) || R * C >= (1ll << 31)) {
    set_error("band does not fit shared memory");
    return T213_ERR_UNSUPPORTED;
  }
  const int64_t bbytes = R * C * eb;
  const bool bulk_ok = (((uintptr_t)data | (uint64_t)bbytes) % 16 == 0) && bbytes <= kBandSmemCap / 2;
  if (bulk_ok) {
    const int64_t sbytes = (bbytes + 127) / 128 * 128;
    const int nbuf = (int)std::max<int64_t>(2, std::min<int64_t>(4, (kBandSmemCap - 128) / sbytes));
    const int64_t smem = 128 + nbuf * sbytes;
    const int Q = 16 / eb;
    const bool vec = eb >= 2 && eb <= 8 && (R % Q == 0) && (C % Q == 0);
    int rc = T213_OK;
    int *stw = device_status_word(&rc);
    if (!stw) return rc;
    auto gob = [&](auto EBc, auto VECc) -> int {
      constexpr int EB = decltype(EBc)::value;
      constexpr bool VEC = decltype(VECc)::value;
      auto kern = k_band_bulk<EB, VEC>;
      if (!kernel_attr_once((const void *)kern, smem, 1)) return cuda_status(cudaGetLastError(), "cudaFuncSetAttribute(band bulk)");
      cudaError_t e;
      const int64_t grid = resident_grid(kern, kTileThreads, (size_t)smem, n_bands);
      const uint32_t cq = (uint32_t)std::max<int64_t>(1, C / (16 / EB));
      kern<<<(unsigned)grid, kTileThreads, (size_t)smem, st>>>(data, n_bands, (uint32_t)R, (uint32_t)C, nbuf,
                                                              FastDiv<uint32_t>((uint64_t)C), FastDiv<uint32_t>((uint64_t)R),
                                                              FastDiv<uint32_t>((uint64_t)cq), stw);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_status(e, "k_band_bulk launch");
      if (ls) ls->launches++;
      return T213_OK;
    };
    using TT = std::true_type;
    using FF = std::false_type;
    switch (eb) {
      case 1:
        return vec ? gob(IC<1>{}, TT{}) : gob(IC<1>{}, FF{});
      case 2:
        return vec ? gob(IC<2>{}, TT{}) : gob(IC<2>{}, FF{});
      case 4:
        return vec ? gob(IC<4>{}, TT{}) : gob(IC<4>{}, FF{});
      case 8:
        return vec ? gob(IC<8>{}, TT{}) : gob(IC<8>{}, FF{});
      case 16:
        return gob(IC<16>{}, FF{});
    }
  }
  const uint32_t S = (uint32_t)((C % 2 == 0) ? C + 1 : C);
  auto go = [&](auto EBc) -> int {
    constexpr int EB = decltype(EBc)::value;
    auto kern = k_band_transpose<EB>;
    if (!kernel_attr_once((const void *)kern, smem, 1)) return cuda_status(cudaGetLastError(), "cudaFuncSetAttribute(band)");
    cudaError_t e;
    const int64_t grid = resident_grid(kern, kTileThreads, (size_t)smem, n_bands);
    kern<<<(unsigned)grid, kTileThreads, (size_t)smem, st>>>(data, n_bands, (uint32_t)R, (uint32_t)C, S,
                                                            FastDiv<uint32_t>((uint64_t)C),
                                                            FastDiv<uint32_t>((uint64_t)R));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "k_band_transpose launch");
    if (ls) ls->launches++;
    return T213_OK;
  };
  switch (eb) {
    case 1:
      return go(IC<1>{});
    case 2:
      return go(IC<2>{});
    case 4:
      return go(IC<4>{});
    case 8:
      return go(IC<8>{});
    case 16:
      return go(IC<16>{});
  }
  set_error("unsupported element size");
  return T213_ERR_UNSUPPORTED;
}

}  // namespace t213
