// Single-system assembly, float (mixed precision).  Three kernels, tried in this order:
//  * the persistent row-panel kernel (assembly_panel.cuh): band windows of up to 2 valence and 2 conduction
//    bands, the band overlaps on the tensor cores read straight from tensor memory;
//  * the tile kernel with the overlaps on the tensor cores (assemble_tile_tc, assembly_tc.cuh): one CTA per
//    upper-triangular (k-block, k'-block) tile, tile side 16 k points for windows of up to 4 e-h pairs per k,
//    8 for larger windows;
//  * the same tile on the CUDA cores (assemble_tile, assembly_tile.cuh).
// XATU_ASSEMBLY_CUDA_CORE=1 in the environment selects the last, XATU_ASSEMBLY_TILE_TC=1 the second.
#include <cstdlib>

#include "assembly_panel.cuh"
#include "engine.h"

template <typename T, int NV, int NC, int NA, bool MIXED, int TK>
__global__ void __launch_bounds__(TK * TK)
bse_assemble_tile_kernel(AsmParams p, AsmInputs in, AsmOutputs out, int nblk) {
  assemble_tile<T, NV, NC, NA, MIXED, TK>(p, in, out, nblk, blockIdx.x);
}

template <int NV, int NC, int NA, int TK>
__global__ void __launch_bounds__(asm_tc_threads(TK))
bse_assemble_tile_tc_kernel(AsmParams p, AsmInputs in, AsmOutputs out, int nblk) {
  assemble_tile_tc<NV, NC, NA, TK>(p, in, out, nblk, blockIdx.x);
}

template <int NV, int NC, int NA>
static cudaError_t launch_tile_tc(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  constexpr int TK = (NV * NC <= 4) ? 16 : 8;
  // one M = 128 product per overlap: atoms x k points x bands must fit its rows
  if constexpr (NA * TK * NC > 128 || NA * TK * NV > 128 || 2 * TK * (NV + NC) > 256) {
    return cudaErrorNotSupported;
  } else {
  const int nblk = (p.nk + TK - 1) / TK;
  const int ntiles = nblk * (nblk + 1) / 2;
  const AsmTcGeom g = asm_tc_geom<NV, NC, NA, TK>(p.norb);
  if (g.KP > XATU_ASM_TC_KPMAX || g.bytes > 200 * 1024) return cudaErrorNotSupported;
  const AsmTcImage im = asm_tc_image<NV, NC, NA, TK>(g);
  if (!in.tc_ops || in.tc_ops_bytes < (size_t)nblk * im.block) return cudaErrorNotSupported;
  // operand images of every k block, then the tiles
  const long long items = (long long)nblk * TK * (NV + NC) * (g.KP / 8);
  asm_tc_format_kernel<NV, NC, NA, TK><<<(unsigned)((items + 255) / 256), 256, 0, s>>>(p, in, nblk);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  auto kern = bse_assemble_tile_tc_kernel<NV, NC, NA, TK>;
  e = xatu_raise_smem_limit((const void*)kern, g.bytes);
  if (e != cudaSuccess) return e;
  kern<<<ntiles, asm_tc_threads(TK), g.bytes, s>>>(p, in, out, nblk);
  return cudaGetLastError();
  }
}

static int panel_num_sms() {
  static int cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

// Row-panel kernel: operand images, FP32 table and k coordinates, the persistent assembly, the diagonal blocks'
// lower triangles.
template <int NV, int NC, int NA>
static cudaError_t launch_panel(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  if constexpr (!PanelShape<NV, NC, NA>::SUPPORTED) {
    return cudaErrorNotSupported;
  } else {
    AsmPanelGeom g;
    if (!asm_panel_geom<NV, NC, NA>(p, g)) return cudaErrorNotSupported;
    if (!in.tc_ops || in.tc_ops_bytes < g.bytes) return cudaErrorNotSupported;
    auto kern = bse_assemble_panel_kernel<NV, NC, NA>;
    // the register split of the warpgroups needs the full launch allotment (setmaxnreg.inc would wait forever
    // on a smaller pool)
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)kern);
    if (e != cudaSuccess) return e;
    if (fa.numRegs != XATU_PANEL_REGS_LAUNCH) return cudaErrorNotSupported;
    e = xatu_raise_smem_limit((const void*)kern, g.smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(in.tc_ops + g.img_F, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    asm_panel_format_kernel<NV, NC, NA><<<4 * panel_num_sms(), 256, 0, s>>>(p, in, g);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int grid = g.total < panel_num_sms() ? g.total : panel_num_sms();
    // the panel kernel and the mirror are launched chained (each waits for its predecessor grid at entry)
    e = xatu_launch_chained(kern, dim3(grid), dim3(XATU_PANEL_THREADS), g.smem, s, p, in, out, g);
    if (e != cudaSuccess) return e;
    const unsigned nd = (unsigned)((p.N + XATU_KBLOCK - 1) / XATU_KBLOCK);
    return xatu_launch_chained(asm_diag_mirror_kernel, dim3(nd, 10), dim3(32, 8), 0, s,
                               reinterpret_cast<unsigned*>(out.Khi), reinterpret_cast<unsigned*>(out.Klo), p.N,
                               p.ldk);
  }
}

template <int NV, int NC, int NA>
static size_t tc_scratch(const AsmParams& p) {
  constexpr int TK = (NV * NC <= 4) ? 16 : 8;
  size_t bytes = 0;
  if constexpr (!(NA * TK * NC > 128 || NA * TK * NV > 128 || 2 * TK * (NV + NC) > 256)) {
    const AsmTcGeom g = asm_tc_geom<NV, NC, NA, TK>(p.norb);
    if (g.KP <= XATU_ASM_TC_KPMAX) bytes = (size_t)((p.nk + TK - 1) / TK) * asm_tc_image<NV, NC, NA, TK>(g).block;
  }
  AsmPanelGeom pg;
  if (asm_panel_geom<NV, NC, NA>(p, pg) && pg.bytes > bytes) bytes = pg.bytes;
  return bytes;
}

size_t xatu_assembly_tc_scratch_bytes(const AsmParams& p) {
#define XATU_CASE(NVv, NCv)                                 \
  if (p.nv == NVv && p.nc == NCv) {                         \
    if (p.na == 1) return tc_scratch<NVv, NCv, 1>(p);       \
    if (p.na == 2) return tc_scratch<NVv, NCv, 2>(p);       \
    if (p.na == 3) return tc_scratch<NVv, NCv, 3>(p);       \
    if (p.na == 4) return tc_scratch<NVv, NCv, 4>(p);       \
  }
  XATU_CASE(1, 1)
  XATU_CASE(1, 2)
  XATU_CASE(1, 3)
  XATU_CASE(2, 1)
  XATU_CASE(2, 2)
  XATU_CASE(2, 3)
  XATU_CASE(3, 1)
  XATU_CASE(3, 2)
  XATU_CASE(3, 3)
#undef XATU_CASE
  return 0;
}

template <typename T, int NV, int NC, int NA, bool MIXED>
static cudaError_t launch_tile(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s) {
  constexpr int TK = (NV * NC <= 4) ? 16 : 8;
  const int nblk = (p.nk + TK - 1) / TK;
  const int ntiles = nblk * (nblk + 1) / 2;
  constexpr int TR = TK * NV * NC;
  const size_t smem = (2 * (size_t)(NV + NC) * p.norb * (TK + 1) + (size_t)TR * (TR + 1) +
                       (p.exchange ? 2 * (size_t)TR * NA : 0)) *
                      sizeof(cplx<T>);
  if (smem > 200 * 1024) return cudaErrorNotSupported;
  auto kern = bse_assemble_tile_kernel<T, NV, NC, NA, MIXED, TK>;
  cudaError_t e = xatu_raise_smem_limit((const void*)kern, smem);
  if (e != cudaSuccess) return e;
  kern<<<ntiles, TK * TK, smem, s>>>(p, in, out, nblk);
  return cudaGetLastError();
}

// Launches the tile kernel of the band-window class of p; *launched = false when the class has none.
cudaError_t xatu_dispatch_tile_f32(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out, cudaStream_t s,
                          bool* launched, bool* tensor_cores, bool* panel) {
  *launched = true;
  *tensor_cores = false;
  *panel = false;
  const char* cc = std::getenv("XATU_ASSEMBLY_CUDA_CORE");
  const bool allow_tc = !(cc && cc[0] == '1');
  const char* tt = std::getenv("XATU_ASSEMBLY_TILE_TC");
  const bool allow_panel = allow_tc && !(tt && tt[0] == '1');
  // the row-panel kernel, then the tensor-core tile; cudaErrorNotSupported (band window, orbital basis or
  // staging too large) falls back
#define XATU_TRY_TC(NVt, NCt, NAt)                                                           \
  if (allow_panel) {                                                                         \
    cudaError_t e = launch_panel<NVt, NCt, NAt>(p, in, out, s);                               \
    if (e != cudaErrorNotSupported) {                                                        \
      *tensor_cores = e == cudaSuccess;                                                      \
      *panel = e == cudaSuccess;                                                             \
      return e;                                                                              \
    }                                                                                        \
  }                                                                                          \
  if (allow_tc) {                                                                            \
    cudaError_t e = launch_tile_tc<NVt, NCt, NAt>(p, in, out, s);                             \
    if (e != cudaErrorNotSupported) {                                                        \
      *tensor_cores = e == cudaSuccess;                                                      \
      return e;                                                                              \
    }                                                                                        \
  }
#define XATU_CASE(NVv, NCv)                                                                  \
  if (p.nv == NVv && p.nc == NCv) {                                                          \
    if (p.na == 1) { XATU_TRY_TC(NVv, NCv, 1) return launch_tile<float, NVv, NCv, 1, true>(p, in, out, s); } \
    if (p.na == 2) { XATU_TRY_TC(NVv, NCv, 2) return launch_tile<float, NVv, NCv, 2, true>(p, in, out, s); } \
    if (p.na == 3) { XATU_TRY_TC(NVv, NCv, 3) return launch_tile<float, NVv, NCv, 3, true>(p, in, out, s); } \
    if (p.na == 4) { XATU_TRY_TC(NVv, NCv, 4) return launch_tile<float, NVv, NCv, 4, true>(p, in, out, s); } \
  }
  XATU_CASE(1, 1)
  XATU_CASE(1, 2)
  XATU_CASE(1, 3)
  XATU_CASE(2, 1)
  XATU_CASE(2, 2)
  XATU_CASE(2, 3)
  XATU_CASE(3, 1)
  XATU_CASE(3, 2)
  XATU_CASE(3, 3)
#undef XATU_CASE
#undef XATU_TRY_TC
  *launched = false;
  return cudaSuccess;
}
