// sqg_inst_multi.cu -- the multi-size ensemble passes (one launch over the
// members and scalars of the size classes N = 128, 256, 512).
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {

template <typename T, int L>
constexpr bool multi_row_ok() {
  return rows_per_cta<T, L>() * row_group<T, L>() == kMultiRowThreads;
}
template <typename T, int L>
constexpr bool multi_col_ok() {
  return pairs_per_cta<T, L>() * col_group<T, L>() == kMultiColThreads && col_nbuf<T, L>() == 4;
}
static_assert(multi_row_ok<float, 7>() && multi_row_ok<float, 8>() && multi_row_ok<float, 9>(), "row shapes");
static_assert(multi_row_ok<double, 7>() && multi_row_ok<double, 8>() && multi_row_ok<double, 9>(), "row shapes");
static_assert(multi_col_ok<float, 7>() && multi_col_ok<float, 8>() && multi_col_ok<float, 9>(), "column shapes");
static_assert(multi_col_ok<double, 7>() && multi_col_ok<double, 8>() && multi_col_ok<double, 9>(), "column shapes");

__device__ __forceinline__ const MultiSeg& find_seg(const MultiArgs& ma, int& entity, int& tile) {
  int g = 0;
  while (g + 1 < ma.nseg && (int)blockIdx.x >= ma.seg[g + 1].start) ++g;
  const MultiSeg& sg = ma.seg[g];
  const int local = (int)blockIdx.x - sg.start;
  entity = local / sg.tiles;
  tile = local - entity * sg.tiles;
  return sg;
}

// compile-time launch shapes of class L (evaluated in host context)
template <typename T, int L>
struct MultiShape {
  static constexpr int R = row_radix<T, L>(), RPC = rows_per_cta<T, L>(), DEPTH = row_depth<T, L>(),
                       NFX = row_nfx<T, L>();
  static constexpr int CR = col_radix<T, L>(), NP = pairs_per_cta<T, L>(), NBUF = col_nbuf<T, L>();
};
template <typename T, int L>
__device__ __forceinline__ void row_multi_body(const KP& kp, const RowArgs& a, int tile) {
  using S = MultiShape<T, L>;
  row_body<T, L, S::R, S::RPC, S::DEPTH, S::NFX>(kp, a, tile);
}
template <typename T, int L>
__device__ __forceinline__ void col_multi_body(const KP& kp, const ColArgs& a, int tile, int ntiles) {
  using S = MultiShape<T, L>;
  col_body<T, L, S::CR, S::NP, S::NBUF>(kp, a, tile, ntiles);
}

template <typename T>
constexpr int kMultiRowMinBlocks = 65536 / (kMultiRowThreads * (sizeof(T) == 4 ? 64 : 128));
template <typename T>
__global__ void __launch_bounds__(kMultiRowThreads, kMultiRowMinBlocks<T>)
k_row_multi(const MultiArgs ma) {
  pdl_wait();
  int e, tile;
  const MultiSeg& sg = find_seg(ma, e, tile);
  // read in place (a local copy would be indexed dynamically and spill)
  const KP& kp = sg.kps[e];
  const RowArgs& a = reinterpret_cast<const RowArgs*>(sg.args)[e];
  switch (sg.log2n) {
    case 7: row_multi_body<T, 7>(kp, a, tile); break;
    case 8: row_multi_body<T, 8>(kp, a, tile); break;
    case 9: row_multi_body<T, 9>(kp, a, tile); break;
    default: break;
  }
}

template <typename T>
constexpr int kMultiColMinBlocks = 65536 / (kMultiColThreads * (sizeof(T) == 4 ? 128 : 168));
template <typename T>
__global__ void __launch_bounds__(kMultiColThreads, kMultiColMinBlocks<T>)
k_col_multi(const MultiArgs ma) {
  pdl_wait();
  int e, tile;
  const MultiSeg& sg = find_seg(ma, e, tile);
  const KP& kp = sg.kps[e];
  const ColArgs& a = reinterpret_cast<const ColArgs*>(sg.args)[e];
  switch (sg.log2n) {
    case 7: col_multi_body<T, 7>(kp, a, tile, sg.tiles); break;
    case 8: col_multi_body<T, 8>(kp, a, tile, sg.tiles); break;
    case 9: col_multi_body<T, 9>(kp, a, tile, sg.tiles); break;
    default: break;
  }
}

template <typename T>
size_t multi_row_smem() {
  size_t m = row_smem<T, 7>();
  if (row_smem<T, 8>() > m) m = row_smem<T, 8>();
  if (row_smem<T, 9>() > m) m = row_smem<T, 9>();
  return m;
}
template <typename T>
size_t multi_col_smem() {
  size_t m = col_smem<T, 7>();
  if (col_smem<T, 8>() > m) m = col_smem<T, 8>();
  if (col_smem<T, 9>() > m) m = col_smem<T, 9>();
  return m;
}

template <typename T>
cudaError_t launch_row_multi(const MultiArgs& ma, int blocks, cudaStream_t st) {
  return launch_pdl(k_row_multi<T>, dim3(blocks), dim3(kMultiRowThreads), multi_row_smem<T>(), st, ma);
}
template <typename T>
cudaError_t launch_col_multi(const MultiArgs& ma, int blocks, cudaStream_t st) {
  return launch_pdl(k_col_multi<T>, dim3(blocks), dim3(kMultiColThreads), multi_col_smem<T>(), st, ma);
}
template <typename T>
cudaError_t set_multi_attrs() {
  cudaError_t e = cudaFuncSetAttribute(k_row_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)multi_row_smem<T>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_col_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)multi_col_smem<T>());
}
template <typename T>
int multi_row_tiles(int log2n) {
  switch (log2n) {
    case 7: return (64 + 1 + rows_per_cta<T, 7>() - 1) / rows_per_cta<T, 7>();
    case 8: return (128 + 1 + rows_per_cta<T, 8>() - 1) / rows_per_cta<T, 8>();
    case 9: return (256 + 1 + rows_per_cta<T, 9>() - 1) / rows_per_cta<T, 9>();
    default: return 0;
  }
}
template <typename T>
int multi_col_tiles(int log2n) {
  switch (log2n) {
    case 7: return 128 / (2 * pairs_per_cta<T, 7>());
    case 8: return 256 / (2 * pairs_per_cta<T, 8>());
    case 9: return 512 / (2 * pairs_per_cta<T, 9>());
    default: return 0;
  }
}

template cudaError_t launch_row_multi<float>(const MultiArgs&, int, cudaStream_t);
template cudaError_t launch_row_multi<double>(const MultiArgs&, int, cudaStream_t);
template cudaError_t launch_col_multi<float>(const MultiArgs&, int, cudaStream_t);
template cudaError_t launch_col_multi<double>(const MultiArgs&, int, cudaStream_t);
template cudaError_t set_multi_attrs<float>();
template cudaError_t set_multi_attrs<double>();
template int multi_row_tiles<float>(int);
template int multi_row_tiles<double>(int);
template int multi_col_tiles<float>(int);
template int multi_col_tiles<double>(int);

}  // namespace sqg
