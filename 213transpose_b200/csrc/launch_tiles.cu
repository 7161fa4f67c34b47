// Launchers of the square-block tile swaps and of the band transposes.
#include <algorithm>

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
