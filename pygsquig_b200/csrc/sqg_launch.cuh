// sqg_launch.cuh -- launch shapes of the row and column passes and the
// per-size launch functions.
//
// The launch functions are templates over the precision T and log2(N).  Their
// definitions (which instantiate the pass kernels) are compiled only by the
// translation units sqg_inst_*.cu, each for a range of sizes, so that the
// kernel instantiations build in parallel; sqg_capi.cu sees the declarations
// and dispatches on log2(N) at run time.
#pragma once
#include <cstring>

#include "sqg_kernels.cuh"

namespace sqg {

// ---- compile-time launch shapes ----
// Radix of the group FFTs.  Column pass: 16 for float grids with N >= 2048
// (groups of N/16 threads, one exchange pass fewer, two 256-thread blocks per
// SM; measured at N = 4096: 370 -> 271 us per launch); row pass: 8 at those
// sizes (radix 16 with two exchange buffers made the fused stage pass slower,
// 384 -> 508 us, because its stage update walks 16 prefetched chunks per
// thread).  Grids with 128 <= N <= 2048: radix-4 row pass (twice the threads
// per transform at 64 registers in single precision, 128 in double; at
// N <= 1024 the pass is one wave of blocks bound by each block's latency:
// FP32 N = 1024 row passes 31 -> 20 us, FP64 52 -> 36 us; N = 2048 step
// FP32 0.64 -> 0.57 ms, FP64 1.36 -> 1.19 ms; at N = 4096 it was slower,
// 315 -> 357 us); the column pass stays radix 8 there (radix 4 took
// 23 -> 30 us at N = 1024 in single precision, 34 -> 39 us in double).
template <typename T, int L>
constexpr int col_radix() { return (sizeof(T) == 4 && L >= 11) ? 16 : 8; }
template <typename T, int L>
constexpr int row_radix() { return (L >= 7 && L <= 11) ? 4 : 8; }
// The last stage of a step (no inverse transforms) uses the same radix, so
// that a step and a replayed multistep step round identically.
template <typename T, int L>
constexpr int rowx_radix() { return row_radix<T, L>(); }
template <typename T, int L>
constexpr int rowx_group() { return (1 << L) / rowx_radix<T, L>(); }
template <typename T, int L>
constexpr int rowx_rpc() { return rowx_group<T, L>() >= 128 ? 1 : 128 / rowx_group<T, L>(); }
template <typename T, int L>
constexpr int row_group() { return (1 << L) / row_radix<T, L>(); }
template <typename T, int L>
constexpr int col_group() { return (1 << L) / col_radix<T, L>(); }
template <typename T, int L>
constexpr int rows_per_cta() { return row_group<T, L>() >= 128 ? 1 : 128 / row_group<T, L>(); }
template <typename T, int L>
constexpr int pairs_per_cta() {
  constexpr int g = col_group<T, L>();
  constexpr int cap = (1 << L) / 2 < 16 ? (1 << L) / 2 : 16;
  // radix 16: up to two column pairs (four columns fill the 32-byte sectors
  // of each row's gather); the autotuner picks one or two
  if (col_radix<T, L>() == 16) return 2;
  return g >= 256 ? 1 : (256 / g > cap ? cap : 256 / g);
}
// Four resident field buffers per column pair when they fit in 150 KB; the
// radix-16 column pass (FP32, N >= 2048) keeps two (two rounds of two fields,
// about 35 KB a buffer: one or two column pairs per block as the autotuner
// chose, 70 or 140 KB).
template <typename T, int L>
constexpr int col_nbuf() {
  return col_radix<T, L>() == 16 ? 2
         : (size_t)pairs_per_cta<T, L>() * 4 * ColBuf<(1 << L), col_radix<T, L>()>::SZ *
                       sizeof(typename Cplx<T>::type) <= 150 * 1024 ? 4 : 2;
}
// Fields the row pass transforms together (row_body's NFX): four (one
// exchange buffer each) when their buffers fit in 150 KB, else two (two
// rounds); two for a radix-4 or radix-16 row pass.  FP32 at N = 4096 takes
// two at a time with theta_{s+1} parked in shared memory (NFX = 6) at 64
// registers, two 512-thread blocks per SM (measured against four fields from
// registers at one block per SM: theta stage pass 332 -> 289 us; scalar
// stage pass 221 -> 202 us against one field at a time).
template <typename T, int L>
constexpr int row_nfx() {
  if (sizeof(T) == 4 && L == 12) return 6;
  return row_radix<T, L>() != 8 ? 2
         : (size_t)rows_per_cta<T, L>() * 4 * spad_size<row_radix<T, L>()>(1 << L) * sizeof(typename Cplx<T>::type) <=
                   150 * 1024 ? 4 : 2;
}
template <typename T, int L, int NFX = row_nfx<T, L>()>
constexpr size_t row_base_smem() {
  return (size_t)rows_per_cta<T, L>() * (NFX > 0 ? nfx_fields(NFX) : 1) * spad_size<row_radix<T, L>()>(1 << L) *
         sizeof(typename Cplx<T>::type);
}
template <typename T, int L>
constexpr size_t row_pf_bytes(int depth) {
  return (size_t)rows_per_cta<T, L>() * depth * 4 * row_group<T, L>() * sizeof(typename Cplx<T>::type);
}
// Prefetch depth of the row pass: among R, R/2, R/4 and 1 chunks, the one
// that lets the most blocks share an SM (the register budget's block count,
// 227 KB of shared memory per SM with 1 KB reserved per block, at most 220 KB
// per block), the deepest among equals: occupancy first, then prefetch depth.
template <typename T, int L, int NFX = row_nfx<T, L>()>
constexpr int row_occupancy(int depth) {
  constexpr int by_regs = row_min_blocks<T, row_radix<T, L>(), NFX>(rows_per_cta<T, L>() * row_group<T, L>());
  const size_t smem = row_base_smem<T, L, NFX>() + row_pf_bytes<T, L>(depth);
  if (smem > 220 * 1024) return 0;
  const int by_smem = (int)((227 * 1024) / (smem + 1024));
  return by_smem < by_regs ? by_smem : by_regs;
}
template <typename T, int L, int NFX = row_nfx<T, L>()>
constexpr int row_depth() {
  constexpr int R = row_radix<T, L>();
  int best = 1, occ = row_occupancy<T, L, NFX>(1);
  for (int d = 2; d <= R; d *= 2) {
    const int o = row_occupancy<T, L, NFX>(d);
    if (o >= occ && o > 0) { occ = o; best = d; }
  }
  // the parked passes keep theta_{s+1} in the staging slots (N elements)
  if (nfx_park(NFX))
    while (best < R && best * 4 * row_group<T, L>() < (1 << L)) best *= 2;
  return best;
}
template <typename T, int L, int NFX = row_nfx<T, L>()>
size_t row_smem() { return row_base_smem<T, L, NFX>() + row_pf_bytes<T, L>(row_depth<T, L, NFX>()); }
// The stage pass without inverse transforms (the last stage of a step): one
// exchange buffer per row pair, registers as row_min_blocks<.., 0>; prefetch
// depth again occupancy first.
template <typename T, int L>
constexpr size_t rowx_smem(int depth) {
  return (size_t)rowx_rpc<T, L>() * (spad_size<rowx_radix<T, L>()>(1 << L) + depth * 4 * rowx_group<T, L>()) *
         sizeof(typename Cplx<T>::type);
}
template <typename T, int L>
constexpr int rowx_occupancy(int depth) {
  constexpr int by_regs = row_min_blocks<T, rowx_radix<T, L>(), 0>(rowx_rpc<T, L>() * rowx_group<T, L>());
  const size_t smem = rowx_smem<T, L>(depth);
  if (smem > 220 * 1024) return 0;
  const int by_smem = (int)((227 * 1024) / (smem + 1024));
  return by_smem < by_regs ? by_smem : by_regs;
}
template <typename T, int L>
constexpr int rowx_depth() {
  constexpr int R = rowx_radix<T, L>();
  int best = 1, occ = rowx_occupancy<T, L>(1);
  for (int d = 2; d <= R; d *= 2) {
    const int o = rowx_occupancy<T, L>(d);
    if (o >= occ && o > 0) { occ = o; best = d; }
  }
  return best;
}
template <typename T, int L>
size_t col_smem() {  // per column pair: NBUF buffers
  return (size_t)pairs_per_cta<T, L>() * col_nbuf<T, L>() * ColBuf<(1 << L), col_radix<T, L>()>::SZ *
         sizeof(typename Cplx<T>::type);
}


template <typename T, int L> cudaError_t launch_row_t(const KP& kp, const RowArgs& a, cudaStream_t st);
template <typename T, int L>
cudaError_t launch_col_t(const KP& kp, const ColArgs& a, cudaStream_t st, bool ring_only, const CUtensorMap* tm);
template <typename T, int L> cudaError_t shape_max_t(int* rpc, int* np);
template <typename T, int L> cudaError_t set_attrs_t();
template <typename T, int L> cudaError_t launch_row_batch_t(const KP* kps, const RowArgs* as, int members, cudaStream_t st);
template <typename T, int L> cudaError_t launch_col_batch_t(const KP* kps, const ColArgs* as, int members, cudaStream_t st);
template <typename T, int L> cudaError_t set_batch_attrs_t();

// ---- multi-size ensemble passes ----
// One launch covers every entity (theta of a member, or one passive scalar)
// of several size classes.  The blocks are laid out by segment: segment g
// holds the entities of one class and one kind, tiles blocks per entity from
// block seg[g].start on; a block finds its segment, entity and tile and runs
// the single-field pass body of its class.  The classes N = 128, 256, 512
// share the block shapes (128-thread row blocks, 256-thread column blocks),
// so one launch configuration serves them all.
struct MultiSeg {
  int start;         // first block of the segment
  int tiles;         // blocks per entity
  int log2n;         // size class
  int pad;
  const KP* kps;     // per entity
  const void* args;  // RowArgs[] or ColArgs[] per entity
};
constexpr int kMultiSegs = 8;
struct MultiArgs {
  int nseg;
  int pad;
  MultiSeg seg[kMultiSegs];
};
constexpr int kMultiLo = 7, kMultiHi = 9;  // log2 N of the classes a multi-size launch serves
constexpr int kMultiRowThreads = 128, kMultiColThreads = 256;
template <typename T> cudaError_t launch_row_multi(const MultiArgs& ma, int blocks, cudaStream_t st);
template <typename T> cudaError_t launch_col_multi(const MultiArgs& ma, int blocks, cudaStream_t st);
template <typename T> cudaError_t set_multi_attrs();
// row pairs (column pairs) per block of class log2n in a multi-size launch
template <typename T> int multi_row_tiles(int log2n);
template <typename T> int multi_col_tiles(int log2n);

#ifdef SQG_LAUNCH_DEFS
// Launch shapes: a.rpc row pairs per CTA of the row pass (a.np column pairs
// per CTA of the column pass), a power-of-two divisor of the compiled maximum;
// shared memory scales with it.  Results do not depend on the shape (every
// row and column transform is computed the same way); only the number and
// size of the CTAs change.
// The row and column passes are launched with programmatic dependent launch
// (pdl.cuh): the next pass's launch overlaps the tail of the current one.
// The stage passes of theta and of the scalars run instances compiled for
// their modes alone (RowInst: N = 4096 FP32 theta stage pass 290 -> 282 us,
// scalar stage pass 193 -> 184 us) and, at N >= 2048, for their stage too
// (theta 282 -> 268 us, scalars 184 -> 172 us);
// the other row passes run the instance that reads its modes from the
// arguments.
template <typename T, int L>
constexpr bool row_stage_insts() { return L >= 11; }
constexpr int row_inst(int rmode, int fmode) {
  if (rmode == RM_P1)
    return fmode == FM_THETA ? RI_THETA_P1 : (fmode == FM_SCAL ? RI_SCAL_P1 : (fmode == FM_VEL ? RI_VEL_P1 : RI_ANY));
  return rmode != RM_STAGE ? RI_ANY : (fmode == FM_THETA ? RI_THETA_STAGE : (fmode == FM_SCAL ? RI_SCAL_STAGE : RI_ANY));
}
template <typename T, int L, int RI>
cudaError_t launch_row_i(const KP& kp, const RowArgs& a, cudaStream_t st) {
  constexpr int N = 1 << L, RPC = rows_per_cta<T, L>();
  if constexpr (ri_stage(RI) == 0 && ri_rmode(RI) != RM_P1) {
    if (a.rmode == RM_STAGE && !a.do_p1) {  // last stage: its own radix, the compiled launch shape
      constexpr int RPCX = rowx_rpc<T, L>();
      RowArgs ax = a;
      ax.rpc = 0;
      return launch_pdl(k_row<T, L, rowx_radix<T, L>(), RPCX, rowx_depth<T, L>(), 0, RI>,
                        dim3((N / 2 + 1 + RPCX - 1) / RPCX), dim3(RPCX * rowx_group<T, L>()),
                        rowx_smem<T, L>(rowx_depth<T, L>()), st, kp, ax);
    }
  }
  const int rpc = a.rpc > 0 ? a.rpc : RPC;
  const int grid = (N / 2 + 1 + rpc - 1) / rpc;
  return launch_pdl(k_row<T, L, row_radix<T, L>(), RPC, row_depth<T, L>(), row_nfx<T, L>(), RI>, dim3(grid),
                    dim3(rpc * row_group<T, L>()), row_smem<T, L>() / RPC * rpc, st, kp, a);
}
template <typename T, int L, int RI0>
cudaError_t launch_row_stage_i(const KP& kp, const RowArgs& a, cudaStream_t st) {
  switch (a.stage) {
    case 1: return launch_row_i<T, L, RI0>(kp, a, st);
    case 2: return launch_row_i<T, L, RI0 + 1>(kp, a, st);
    case 3: return launch_row_i<T, L, RI0 + 2>(kp, a, st);
    default: return launch_row_i<T, L, RI0 + 3>(kp, a, st);
  }
}
template <typename T, int L>
cudaError_t launch_row_t(const KP& kp, const RowArgs& a, cudaStream_t st) {
  const int ri = row_inst(a.rmode, a.fmode);
  if constexpr (row_stage_insts<T, L>()) {
    if (a.do_p1 && a.stage >= 1 && a.stage <= 4) {
      if (ri == RI_THETA_STAGE) return launch_row_stage_i<T, L, RI_THETA_S1>(kp, a, st);
      if (ri == RI_SCAL_STAGE) return launch_row_stage_i<T, L, RI_SCAL_S1>(kp, a, st);
    }
  }
  switch (ri) {
    case RI_THETA_STAGE: return launch_row_i<T, L, RI_THETA_STAGE>(kp, a, st);
    case RI_SCAL_STAGE: return launch_row_i<T, L, RI_SCAL_STAGE>(kp, a, st);
    case RI_THETA_P1: return launch_row_i<T, L, RI_THETA_P1>(kp, a, st);
    case RI_SCAL_P1: return launch_row_i<T, L, RI_SCAL_P1>(kp, a, st);
    case RI_VEL_P1: return launch_row_i<T, L, RI_VEL_P1>(kp, a, st);
    default: return launch_row_i<T, L, RI_ANY>(kp, a, st);
  }
}
// Column passes of theta and of the scalars run instances compiled for their
// mode alone (fewer registers live, fewer spills: N = 4096 FP32 theta column
// pass 212 -> 204 us, scalar column pass 149 -> 134 us); the other modes run
// the instance that chooses the mode at run time (an instance for the
// velocity pass alone was slower, 90 -> 92 us).
// Field buffers per column pair of a mode instance: theta's two-round pass at
// N = 4096 keeps a third, which receives round 2's first field during round 1
// (FP32 205 -> 197 us, FP64 532 -> 518 us).
template <typename T, int L, int CMX>
constexpr int col_nbuf_m() { return (CMX == CM_THETA && col_nbuf<T, L>() == 2 && L == 12) ? 3 : col_nbuf<T, L>(); }
template <typename T, int L, int CMX>
size_t col_smem_m() { return col_smem<T, L>() / col_nbuf<T, L>() * col_nbuf_m<T, L, CMX>(); }
// tm (host copy): the tensor map of the field stack a.xh, passed as the
// kernel's grid-constant parameter (null: the passes gather with cp.async).
template <typename T, int L, int CMX>
cudaError_t launch_col_m(const KP& kp, const ColArgs& a, cudaStream_t st, int grid, int np, const CUtensorMap* tm) {
  constexpr int NP = pairs_per_cta<T, L>();
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  ColArgs b = a;
  b.tma = 0;
  if (tm && (1 << L) >= kColTmaMinN && a.cmode != CM_SCALV) {
    m = *tm;
    b.tma = 1;
  }
  return launch_pdl(k_col<T, L, col_radix<T, L>(), NP, col_nbuf_m<T, L, CMX>(), CMX>, dim3(grid),
                    dim3(np * col_group<T, L>()), col_smem_m<T, L, CMX>() / NP * np, st, kp, b, m);
}
template <typename T, int L>
cudaError_t launch_col_t(const KP& kp, const ColArgs& a, cudaStream_t st, bool ring_only, const CUtensorMap* tm) {
  constexpr int N = 1 << L, NP = pairs_per_cta<T, L>();
  const int np = a.np > 0 ? a.np : NP;
  const int grid = ring_only ? 1 : N / (2 * np) + (a.ring_cta ? 1 : 0);
  if (a.cmode == CM_THETA) return launch_col_m<T, L, CM_THETA>(kp, a, st, grid, np, tm);
  if (a.cmode == CM_SCAL && !a.ring_cta) return launch_col_m<T, L, CM_SCAL>(kp, a, st, grid, np, tm);
  return launch_col_m<T, L, -1>(kp, a, st, grid, np, tm);
}
template <typename T, int L>
cudaError_t shape_max_t(int* rpc, int* np) {
  *rpc = rows_per_cta<T, L>();
  *np = pairs_per_cta<T, L>();
  return cudaSuccess;
}
template <typename T, int L, int RI>
cudaError_t set_row_attrs_i() {
  constexpr int RPC = rows_per_cta<T, L>();
  cudaError_t e = cudaFuncSetAttribute(k_row<T, L, row_radix<T, L>(), RPC, row_depth<T, L>(), row_nfx<T, L>(), RI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem<T, L>());
  if constexpr (ri_stage(RI) == 0 && ri_rmode(RI) != RM_P1) {  // the last-stage kernel: the stage instances
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_row<T, L, rowx_radix<T, L>(), rowx_rpc<T, L>(), rowx_depth<T, L>(), 0, RI>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rowx_smem<T, L>(rowx_depth<T, L>()));
  }
  return e;
}
template <typename T, int L, int RI0>
cudaError_t set_row_stage_attrs_i() {
  cudaError_t e = set_row_attrs_i<T, L, RI0>();
  if (e == cudaSuccess) e = set_row_attrs_i<T, L, RI0 + 1>();
  if (e == cudaSuccess) e = set_row_attrs_i<T, L, RI0 + 2>();
  if (e == cudaSuccess) e = set_row_attrs_i<T, L, RI0 + 3>();
  return e;
}
template <typename T, int L>
cudaError_t set_attrs_t() {
  constexpr int NP = pairs_per_cta<T, L>();
  cudaError_t e = set_row_attrs_i<T, L, RI_ANY>();
  if (e != cudaSuccess) return e;
  e = set_row_attrs_i<T, L, RI_THETA_STAGE>();
  if (e != cudaSuccess) return e;
  e = set_row_attrs_i<T, L, RI_SCAL_STAGE>();
  if (e != cudaSuccess) return e;
  e = set_row_attrs_i<T, L, RI_THETA_P1>();
  if (e != cudaSuccess) return e;
  e = set_row_attrs_i<T, L, RI_SCAL_P1>();
  if (e != cudaSuccess) return e;
  e = set_row_attrs_i<T, L, RI_VEL_P1>();
  if (e != cudaSuccess) return e;
  if constexpr (row_stage_insts<T, L>()) {
    e = set_row_stage_attrs_i<T, L, RI_THETA_S1>();
    if (e != cudaSuccess) return e;
    e = set_row_stage_attrs_i<T, L, RI_SCAL_S1>();
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(k_col<T, L, col_radix<T, L>(), NP, col_nbuf_m<T, L, CM_THETA>(), CM_THETA>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem_m<T, L, CM_THETA>());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_col<T, L, col_radix<T, L>(), NP, col_nbuf<T, L>(), CM_SCAL>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem<T, L>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_col<T, L, col_radix<T, L>(), NP, col_nbuf<T, L>()>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem<T, L>());
}

template <typename T, int L>
cudaError_t launch_row_batch_t(const KP* kps, const RowArgs* as, int members, cudaStream_t st) {
  constexpr int N = 1 << L, RPC = rows_per_cta<T, L>();
  dim3 grid((N / 2 + 1 + RPC - 1) / RPC, members);
  return launch_pdl(k_row_batch<T, L, row_radix<T, L>(), RPC, row_depth<T, L>(), row_nfx<T, L>()>, grid,
                    dim3(RPC * row_group<T, L>()), row_smem<T, L>(), st, kps, as);
}
template <typename T, int L>
cudaError_t launch_col_batch_t(const KP* kps, const ColArgs* as, int members, cudaStream_t st) {
  constexpr int N = 1 << L, NP = pairs_per_cta<T, L>();
  dim3 grid(N / (2 * NP), members);
  return launch_pdl(k_col_batch<T, L, col_radix<T, L>(), NP, col_nbuf<T, L>()>, grid,
                    dim3(NP * col_group<T, L>()), col_smem<T, L>(), st, kps, as);
}
template <typename T, int L>
cudaError_t set_batch_attrs_t() {
  constexpr int RPC = rows_per_cta<T, L>(), NP = pairs_per_cta<T, L>();
  cudaError_t e = cudaFuncSetAttribute(k_row_batch<T, L, row_radix<T, L>(), RPC, row_depth<T, L>(), row_nfx<T, L>()>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem<T, L>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_col_batch<T, L, col_radix<T, L>(), NP, col_nbuf<T, L>()>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem<T, L>());
}

// Explicit instantiation of every launch function for one (T, log2 N).
#define SQG_INSTANTIATE(T, L)                                                                               \
  template cudaError_t launch_row_t<T, L>(const KP&, const RowArgs&, cudaStream_t);                        \
  template cudaError_t launch_col_t<T, L>(const KP&, const ColArgs&, cudaStream_t, bool, const CUtensorMap*); \
  template cudaError_t shape_max_t<T, L>(int*, int*);                                                      \
  template cudaError_t set_attrs_t<T, L>();                                                                \
  template cudaError_t launch_row_batch_t<T, L>(const KP*, const RowArgs*, int, cudaStream_t);             \
  template cudaError_t launch_col_batch_t<T, L>(const KP*, const ColArgs*, int, cudaStream_t);             \
  template cudaError_t set_batch_attrs_t<T, L>();
#endif

}  // namespace sqg
