// closure_conv.cu -- BF16 tensor-core (tcgen05) 3x3 convolution with 64 input
// and 64 output channels for the learned subgrid closure.
//
// Implicit GEMM: M = 128 pixels of one image row (a tile), N = 64 output
// channels, K = 9 taps x 64 input channels (one 64-wide K block per tap).
// Activations are NHWC BF16 with a one-pixel circular halo.  For each of the
// three input rows a tile needs, one TMA box brings 130 consecutive pixels
// (the tile and its two neighbours: 130 rows of 128 bytes, 128B-swizzled)
// into a 1024-byte aligned slab.  The A operand of tap (dy, dx) is the slab of
// row dy read from row dx: the descriptor start moves by dx rows (base offset
// 0: the 128-byte swizzle follows the absolute shared-memory address bits,
// as the TMA wrote them, so a row-shifted start reads the same layout).  Each
// activation byte is fetched three times instead of nine, in 128-byte rows.
// The weights of the 9 taps stay in shared memory (128B-swizzled, K-major)
// for the life of the persistent CTA.
//
// Warp roles (10 warps): warp 0 issues TMA loads, warp 1 allocates TMEM and
// issues the MMAs (one elected thread), warps 2..9 read the FP32 accumulators
// from TMEM (tcgen05.ld; warp w may read lane quarter w % 4, so two warps
// share each quarter and take 32 of the 64 columns each) and run the
// epilogue.  A tile accumulates into four TMEM accumulators, one per 16-wide
// slice of the 64 input channels, so consecutive MMAs never wait on each
// other's result (a single 128 x 64 accumulator chain of 36 short MMAs is
// latency-bound); the epilogue adds the four.  Two such sets alternate so the
// epilogue of tile i overlaps the MMAs of tile i+1 (512 TMEM columns).  The epilogue writes its BF16 outputs into
// 128B-swizzled staging tiles, and one thread stores each tile (and its copy
// on the halo row when the image row is the first or last) with a TMA tensor
// store; the halo-column copies of the first and last pixel of an image row
// are plain stores.  Every mbarrier wait is bounded: on time-out the kernel
// records an error flag, the epilogue warps agree through a barrier
// reduction, and all roles drain and return.
//
// Epilogues:
//   FWD:   z = acc + bias; store z (BF16, unpadded) and gelu(z) (BF16, halo'd)
//   DGRAD: g = acc * gelu'(zprev); store g (BF16, halo'd)
//   LIN:   store acc + bias (FP32, unpadded; plain stores)
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <string>

#include "../../include/sqg_closure.h"
#include "closure_act.cuh"
#include "pdl.cuh"

namespace {

thread_local std::string g_err;
int cfail(int code, const std::string& m) {
  g_err = m;
  return code;
}

constexpr int kTileM = 128;
constexpr int kC = 64;
constexpr int kSlabRows = kTileM + 2;        // pixels of one input-row slab
constexpr int kSlabBytes = kSlabRows * 128;  // 16640 B loaded per slab
constexpr int kSlabStride = 17 * 1024;       // slabs start on 1024-byte boundaries
constexpr int kStages = 6;                   // slabs in flight (two tiles)
constexpr int kBBytes = kC * kC * 2;         // 8 KB per tap
constexpr int kStageTile = kTileM * 128;     // 16 KB staging tile (128 pixels x 64 BF16)
constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr uint32_t kWaitLimit = 1u << 26;

// ---- PTX helpers ------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)));
}
// Bounded wait on the phase parity; returns false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];\n" ::"l"(map),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the staging tiles may be rewritten once the stores issued so far have read them
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the TMA (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// named barrier 1 over the 8 epilogue warps
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 256;\n" ::: "memory"); }
// the same barrier with an OR over the epilogue threads' predicates
__device__ __forceinline__ int epi_sync_or(int pred) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, 256, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(pred)
      : "memory");
  return r;
}
__device__ __forceinline__ uint64_t sw128_desc(const void* smem_tile) {
  // K-major, 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart
  const uint64_t start = (smem_u32(smem_tile) >> 4) & 0x3FFF;
  const uint64_t lbo = 1, sbo = 1024 >> 4;
  return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}
// The same layout read from row `row` of a 1024-byte aligned slab: the start
// moves by row x 128 B; the swizzle phase comes from the address bits.
__device__ __forceinline__ uint64_t slab_desc(const void* slab, int row) {
  const uint32_t addr = smem_u32(slab) + (uint32_t)row * 128u;
  const uint64_t start = (addr >> 4) & 0x3FFF;
  const uint64_t lbo = 1, sbo = 1024 >> 4;
  return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}
// BF16 x BF16 -> FP32, K-major A and B, M = 128, N = 64
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

#define TC_LD32(addr, r)                                                                                      \
  asm volatile(                                                                                               \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"      \
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"                            \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),     \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), \
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),           \
        "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),           \
        "=r"(r[30]), "=r"(r[31])                                                                              \
      : "r"(addr))

struct ConvArgs {
  int B, H, W;            // images, rows, columns (W multiple of 128)
  int mode;               // CLOSURE_EPI_*
  const float* bias;      // [64] (FWD, LIN)
  const __nv_bfloat16* zprev;  // [B][H][W][64] pre-activation of the layer below (DGRAD)
  __nv_bfloat16* out_pad;      // [B][H+2][W+2][64] halo'd output (FWD: gelu(z), DGRAD: g)
  float* out_f32;              // [B][H][W][64] (LIN)
  unsigned* err;
};

// Halo-column copies of 32 BF16 channels (from c0) of pixel (b, y, x), x the
// first or last column: padded column W+1 or 0 of its row, and the corner
// when y is also the first or last row.
__device__ __forceinline__ void store_xhalo(__nv_bfloat16* out, int H, int W, int b, int y, int x, int c0,
                                            const uint4 (&v)[4]) {
  const int Wp = W + 2, Hp = H + 2;
  const int xs = (x == 0) ? W + 1 : 0;
  const int ys[2] = {y + 1, (y == 0) ? H + 1 : (y == H - 1 ? 0 : -1)};
  for (int a = 0; a < 2; ++a) {
    if (ys[a] < 0) continue;
    uint4* dst = reinterpret_cast<uint4*>(out + (((size_t)b * Hp + ys[a]) * Wp + xs) * kC + c0);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[i] = v[i];
  }
}

// Byte offset of 16-byte chunk c of row r in a 128B-swizzled tile.
__device__ __forceinline__ uint32_t sw128_off(int r, int c) { return (uint32_t)r * 128u + (uint32_t)((c ^ (r & 7)) << 4); }

__global__ void __launch_bounds__(kThreads, 1)
k_conv64(const __grid_constant__ CUtensorMap act_map, const __grid_constant__ CUtensorMap w_map,
         const __grid_constant__ CUtensorMap out_map, const __grid_constant__ CUtensorMap z_map, ConvArgs a) {
  pdl_wait();  // the previous kernel's output (this layer's input) is visible after this
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned carve-up
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sB = base;                                   // 9 x 8 KB weights
  unsigned char* sA = sB + 9 * kBBytes;                       // kStages row slabs
  unsigned char* sO = sA + kStages * kSlabStride;             // staging: halo'd output tile
  unsigned char* sZ = sO + kStageTile;                        // staging: pre-activation tile
  uint64_t* bars = reinterpret_cast<uint64_t*>(sZ + kStageTile);
  uint64_t* full = bars;                 // [kStages]
  uint64_t* empty = bars + kStages;      // [kStages]
  uint64_t* acc_full = bars + 2 * kStages;   // [2]
  uint64_t* acc_empty = acc_full + 2;        // [2]
  uint64_t* wbar = acc_empty + 2;            // [1] weights; wbar[2] drain
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(wbar + 3);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_per_row = a.W / kTileM;
  const int n_tiles = a.B * a.H * tiles_per_row;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kEpiWarps);  // one arrive per epilogue warp
    }
    mbar_init(wbar, 1);
    mbar_init(wbar + 2, 1);  // drain barrier of the error path
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      mbar_expect_tx(wbar, 9 * kBBytes);
      for (int t = 0; t < 9; ++t) tma_load_2d(sB + t * kBBytes, &w_map, wbar, 0, t * kC);
      int it = 0;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const int xt = tile % tiles_per_row;
        const int rowi = tile / tiles_per_row;
        const int y = rowi % a.H, b = rowi / a.H;
        for (int dy = 0; dy < 3 && ok; ++dy, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (it >= kStages && !mbar_wait(&empty[s], ph ^ 1)) { ok = false; break; }
          // padded row y + dy, padded columns xt*128 .. xt*128 + 129
          const int q = (b * (a.H + 2) + (y + dy)) * (a.W + 2) + xt * kTileM;
          mbar_expect_tx(&full[s], kSlabBytes);
          tma_load_2d(sA + s * kSlabStride, &act_map, &full[s], 0, q);
        }
      }
      if (!ok) {
        atomicOr(a.err, 1u);
        // drain: wait (bounded) for the copies still in flight
        for (int i = (it > kStages ? it - kStages : 0); i < it; ++i) mbar_wait(&full[i % kStages], (i / kStages) & 1);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      ok = mbar_wait(wbar, 0);
      int it = 0, tcount = 0;
      for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x, ++tcount) {
        const int acc = tcount & 1;
        const uint32_t aph = (tcount >> 1) & 1;
        if (tcount >= 2 && !mbar_wait(&acc_empty[acc], aph ^ 1)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + acc * 256;  // accumulator k at d + 64 k
        for (int dy = 0; dy < 3 && ok; ++dy, ++it) {
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          if (!mbar_wait(&full[s], ph)) { ok = false; break; }
          tc_fence_after();
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            const int t = 3 * dy + dx;
            const uint64_t ad = slab_desc(sA + s * kSlabStride, dx);
            const uint64_t bd = sw128_desc(sB + t * kBBytes);
#pragma unroll
            for (int k = 0; k < 4; ++k)  // K = 16 per MMA: 32 bytes along the 128-byte row
              umma(d + 64 * k, ad + 2 * k, bd + 2 * k, t > 0 ? 1u : 0u);
          }
          umma_commit(&empty[s]);  // frees the slab when these MMAs complete
        }
        umma_commit(&acc_full[acc]);
      }
      if (!ok) {
        atomicOr(a.err, 2u);
        // drain: wait (bounded) until every MMA issued so far has completed
        umma_commit(wbar + 2);
        mbar_wait(wbar + 2, 0);
      }
    }
  } else {
    // ---------------- epilogue (warps 2..9) ----------------
    const int quarter = warp & 3;           // TMEM lane quarter this warp may access
    const int c0 = ((warp - 2) >> 2) * 32;  // its 32 accumulator columns
    const int row = quarter * 32 + lane;    // pixel of the tile
    const bool leader = (warp == 2 && lane == 0);
    float bz[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) bz[i] = (a.mode == CLOSURE_EPI_DGRAD) ? 0.f : a.bias[c0 + i];
    int tcount = 0;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++tcount) {
      const int acc = tcount & 1;
      const uint32_t aph = (tcount >> 1) & 1;
      const int bad = mbar_wait(&acc_full[acc], aph) ? 0 : 1;
      if (leader) bulk_wait_read_all();  // the staging tiles are free again
      if (epi_sync_or(bad)) { ok = false; break; }
      tc_fence_after();
      float v[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = bz[i];
      const uint32_t taddr = tmem + acc * 256 + c0 + ((uint32_t)(quarter * 32) << 16);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        uint32_t r[32];
        TC_LD32(taddr + 64 * k, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] += __uint_as_float(r[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[acc]);
      const int xt = tile % tiles_per_row;
      const int rowi = tile / tiles_per_row;
      const int y = rowi % a.H, b = rowi / a.H;
      const int x = xt * kTileM + row;
      const size_t pix = ((size_t)b * a.H + y) * a.W + x;
      if (a.mode == CLOSURE_EPI_LIN) {
        float4* o = reinterpret_cast<float4*>(a.out_f32 + pix * kC + c0);
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        continue;
      }
      uint4 packed[4];
      if (a.mode == CLOSURE_EPI_FWD) {
        uint4 zp[4];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const __nv_bfloat162 zb = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
          const float2 zr = __bfloat1622float2(zb);  // the stored pre-activation
          reinterpret_cast<__nv_bfloat162*>(zp)[i] = zb;
          reinterpret_cast<__nv_bfloat162*>(packed)[i] = __floats2bfloat162_rn(gelu(zr.x), gelu(zr.y));
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) *reinterpret_cast<uint4*>(sZ + sw128_off(row, (c0 >> 3) + i)) = zp[i];
      } else {  // DGRAD
        const uint4* zsrc = reinterpret_cast<const uint4*>(a.zprev + pix * kC + c0);
        uint4 zq[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) zq[i] = zsrc[i];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float2 z = __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(zq)[i]);
          reinterpret_cast<__nv_bfloat162*>(packed)[i] =
              __floats2bfloat162_rn(v[2 * i] * gelu_grad(z.x), v[2 * i + 1] * gelu_grad(z.y));
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) *reinterpret_cast<uint4*>(sO + sw128_off(row, (c0 >> 3) + i)) = packed[i];
      fence_async_smem();
      epi_sync();
      if (leader) {
        const int Wp = a.W + 2;
        const int xq = xt * kTileM + 1;  // padded column of the tile's first pixel
        tma_store_2d(&out_map, sO, 0, (b * (a.H + 2) + y + 1) * Wp + xq);
        if (y == 0) tma_store_2d(&out_map, sO, 0, (b * (a.H + 2) + a.H + 1) * Wp + xq);
        if (y == a.H - 1) tma_store_2d(&out_map, sO, 0, (b * (a.H + 2)) * Wp + xq);
        if (a.mode == CLOSURE_EPI_FWD) tma_store_2d(&z_map, sZ, 0, (b * a.H + y) * a.W + xt * kTileM);
        bulk_commit();
      }
      if (x == 0 || x == a.W - 1) store_xhalo(a.out_pad, a.H, a.W, b, y, x, c0, packed);
    }
    if (leader) bulk_wait_all();
    if (!ok) atomicOr(a.err, 4u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
  }
}

// ---- weight gradient: D[(tap, ci)][co] = sum_p a[p + off_tap][ci] g[p][co] ----
// M = 128 rows = two taps x 64 input channels (MN-major A: the channel index
// is contiguous in the NHWC rows), N = 64 output channels (MN-major B),
// K = pixels in blocks of 64 of one image row.  Five accumulators (taps
// (0,1) (2,3) (4,5) (6,7) (8,-)) live in TMEM; each persistent CTA sums a
// range of pixel blocks and writes its partial sums; k_wgrad_reduce adds the
// partials in a fixed order.
constexpr int kWStages = 2;
constexpr int kWThreads = 192;  // TMA warp, MMA warp, 4 epilogue warps
constexpr int kWSlot = 64 * kC * 2;             // 8 KB: 64 pixel rows x 64 channels
constexpr int kWStageBytes = 11 * kWSlot;       // 10 activation slots + 1 gradient slot
// MN-major A/B, BF16 -> FP32, M = 128, N = 64
constexpr uint32_t kIdescMN =
    (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint64_t sw128_mn_desc(const void* smem_tile, uint32_t lbo_bytes) {
  // MN-major, 128-byte swizzle: 64 elements (128 B) contiguous along M/N,
  // 8 K-rows per 1024 B atom (SBO); the next 64 M/N elements lbo_bytes away
  const uint64_t start = (smem_u32(smem_tile) >> 4) & 0x3FFF;
  const uint64_t lbo = (lbo_bytes >> 4) & 0x3FFF, sbo = 1024 >> 4;
  return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void umma_mn(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescMN), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

struct WgradArgs {
  int B, H, W;
  float* partials;  // [gridDim.x][5][128][64]
  unsigned* err;
};

__global__ void __launch_bounds__(kWThreads, 1)
k_wgrad64(const __grid_constant__ CUtensorMap act_map, const __grid_constant__ CUtensorMap g_map, WgradArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kWStages * kWStageBytes);
  uint64_t* full = bars;                 // [kWStages]
  uint64_t* empty = bars + kWStages;     // [kWStages]
  uint64_t* acc_full = bars + 2 * kWStages;
  uint64_t* drain = acc_full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bpr = a.W / 64;  // pixel blocks per image row
  const int n_kb = a.B * a.H * bpr;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kWStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      for (int kb = blockIdx.x; kb < n_kb && ok; kb += gridDim.x, ++it) {
        const int s = it % kWStages;
        const uint32_t ph = (it / kWStages) & 1;
        if (it >= kWStages && !mbar_wait(&empty[s], ph ^ 1)) { ok = false; break; }
        const int xb = kb % bpr, rowi = kb / bpr;
        const int y = rowi % a.H, b = rowi / a.H;
        unsigned char* st = base + s * kWStageBytes;
        mbar_expect_tx(&full[s], 10 * kWSlot);
        for (int t = 0; t < 9; ++t) {
          const int dy = t / 3 - 1, dx = t % 3 - 1;
          const int q = (b * (a.H + 2) + (y + 1 + dy)) * (a.W + 2) + (xb * 64 + 1 + dx);
          tma_load_2d(st + t * kWSlot, &act_map, &full[s], 0, q);
        }
        const int qg = (b * (a.H + 2) + (y + 1)) * (a.W + 2) + (xb * 64 + 1);
        tma_load_2d(st + 10 * kWSlot, &g_map, &full[s], 0, qg);
      }
      if (!ok) {
        atomicOr(a.err, 8u);
        for (int i = (it > kWStages ? it - kWStages : 0); i < it; ++i) mbar_wait(&full[i % kWStages], (i / kWStages) & 1);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int it = 0;
      for (int kb = blockIdx.x; kb < n_kb && ok; kb += gridDim.x, ++it) {
        const int s = it % kWStages;
        const uint32_t ph = (it / kWStages) & 1;
        if (!mbar_wait(&full[s], ph)) { ok = false; break; }
        tc_fence_after();
        unsigned char* st = base + s * kWStageBytes;
        // the five accumulators interleave, so consecutive MMAs are independent
#pragma unroll
        for (int k = 0; k < 4; ++k) {  // K = 16 pixel rows = two 1024 B atoms
#pragma unroll
          for (int m = 0; m < 5; ++m) {
            const uint64_t ad = sw128_mn_desc(st + (2 * m) * kWSlot, kWSlot) + 128 * k;
            const uint64_t bd = sw128_mn_desc(st + 10 * kWSlot, kWSlot) + 128 * k;
            umma_mn(tmem + m * 64, ad, bd, (it > 0 || k > 0) ? 1u : 0u);
          }
        }
        umma_commit(&empty[s]);
      }
      umma_commit(acc_full);
      if (!ok) atomicOr(a.err, 16u);
    }
  } else {
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;  // (tap parity, ci)
    if (blockIdx.x < n_kb) {
      if (!mbar_wait(acc_full, 0)) ok = false;
    }
    tc_fence_after();
    float* part = a.partials + (size_t)blockIdx.x * 5 * 128 * 64;
    for (int m = 0; m < 5; ++m) {
      uint32_t r[32];
      float v[64];
      const uint32_t taddr = tmem + m * 64 + ((uint32_t)(quarter * 32) << 16);
      if (ok && blockIdx.x < n_kb) {
        TC_LD32(taddr, r);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
        TC_LD32(taddr + 32, r);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[32 + i] = __uint_as_float(r[i]);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int i = 0; i < 64; ++i) v[i] = 0.f;
      }
      float4* o = reinterpret_cast<float4*>(part + ((size_t)m * 128 + row) * 64);
#pragma unroll
      for (int i = 0; i < 16; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
    if (!ok) atomicOr(a.err, 32u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
  }
}

// dW[t][co][ci] = sum over CTAs of partials[cta][t/2][(t%2)*64 + ci][co]
__global__ void k_wgrad_reduce(const float* __restrict__ partials, int nparts, float* __restrict__ dw) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // over 9 * 64 * 64
  if (idx >= 9 * 64 * 64) return;
  const int t = idx / 4096, co = (idx / 64) % 64, ci = idx % 64;
  const size_t off = ((size_t)(t / 2) * 128 + (t % 2) * 64 + ci) * 64 + co;
  float s = 0.f;
  for (int c = 0; c < nparts; ++c) s += partials[(size_t)c * 5 * 128 * 64 + off];
  dw[idx] = s;
}

// ---- host: tensor maps through the driver entry point -------------------------
typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

PFN_encodeTiled encode_fn() {
  static PFN_encodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiled)p;
  }
  return fn;
}

// rows x 64 BF16 matrix, row stride 128 B, boxes of box_rows x 64, 128B swizzle
bool make_map(CUtensorMap* m, const void* ptr, uint64_t rows, uint32_t box_rows) {
  PFN_encodeTiled f = encode_fn();
  if (!f) return false;
  cuuint64_t dims[2] = {kC, rows};
  cuuint64_t strides[1] = {kC * 2};
  cuuint32_t box[2] = {kC, box_rows};
  cuuint32_t estr[2] = {1, 1};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr size_t kSmemBytes = 1024 + 9 * kBBytes + kStages * kSlabStride + 2 * kStageTile + 256;

}  // namespace

extern "C" {

const char* closure_last_error_string(void) { return g_err.c_str(); }

int closure_conv64(int32_t B, int32_t H, int32_t W, int32_t mode, const void* act_pad, const void* weights,
                   const float* bias, const void* zprev, void* out_pad, void* out_z, float* out_f32,
                   uint32_t* err, int32_t grid, void* stream) {
  if (B <= 0 || H <= 0 || W <= 0 || W % kTileM != 0)
    return cfail(1, "closure_conv64: W must be a positive multiple of 128");
  if (!act_pad || !weights || !err) return cfail(1, "closure_conv64: null pointer");
  if ((uintptr_t)act_pad % 16 || (uintptr_t)weights % 16) return cfail(1, "closure_conv64: pointers must be 16-byte aligned");
  if (mode == CLOSURE_EPI_FWD && (!bias || !out_pad || !out_z)) return cfail(1, "closure_conv64: FWD needs bias, out_pad, out_z");
  if (mode == CLOSURE_EPI_DGRAD && (!zprev || !out_pad)) return cfail(1, "closure_conv64: DGRAD needs zprev, out_pad");
  if (mode == CLOSURE_EPI_LIN && (!bias || !out_f32)) return cfail(1, "closure_conv64: LIN needs bias, out_f32");
  if (mode != CLOSURE_EPI_LIN && (((uintptr_t)out_pad % 16) || (out_z && (uintptr_t)out_z % 16)))
    return cfail(1, "closure_conv64: output pointers must be 16-byte aligned");
  CUtensorMap amap, wmap, omap, zmap;
  const uint64_t prows = (uint64_t)B * (H + 2) * (W + 2);
  if (!make_map(&amap, act_pad, prows, kSlabRows) || !make_map(&wmap, weights, 9 * kC, kC))
    return cfail(2, "closure_conv64: tensor map encoding failed");
  omap = amap;  // unused in LIN mode
  zmap = amap;  // unused unless FWD
  if (mode != CLOSURE_EPI_LIN && !make_map(&omap, out_pad, prows, kTileM))
    return cfail(2, "closure_conv64: tensor map encoding failed (output)");
  if (mode == CLOSURE_EPI_FWD && !make_map(&zmap, out_z, (uint64_t)B * H * W, kTileM))
    return cfail(2, "closure_conv64: tensor map encoding failed (pre-activation)");
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_conv64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) != cudaSuccess)
      return cfail(2, "closure_conv64: shared memory attribute");
    attr = true;
  }
  ConvArgs a;
  a.B = B; a.H = H; a.W = W; a.mode = mode; a.bias = bias;
  a.zprev = (const __nv_bfloat16*)zprev;
  a.out_pad = (__nv_bfloat16*)out_pad;
  a.out_f32 = out_f32;
  a.err = err;
  const int n_tiles = B * H * (W / kTileM);
  int g = grid > 0 ? grid : 148;
  if (g > n_tiles) g = n_tiles;
  cudaError_t e = launch_pdl(k_conv64, dim3(g), dim3(kThreads), kSmemBytes, (cudaStream_t)stream, amap, wmap, omap,
                             zmap, a);
  if (e != cudaSuccess) return cfail(2, std::string("closure_conv64 launch: ") + cudaGetErrorString(e));
  return 0;
}

int closure_wgrad64(int32_t B, int32_t H, int32_t W, const void* act_pad, const void* grad_pad, float* partials,
                    int32_t nparts, float* dw, uint32_t* err, void* stream) {
  if (B <= 0 || H <= 0 || W <= 0 || W % 64 != 0) return cfail(1, "closure_wgrad64: W must be a positive multiple of 64");
  if (!act_pad || !grad_pad || !partials || !dw || !err || nparts <= 0) return cfail(1, "closure_wgrad64: bad arguments");
  CUtensorMap amap, gmap;
  const uint64_t prows = (uint64_t)B * (H + 2) * (W + 2);
  if (!make_map(&amap, act_pad, prows, 64) || !make_map(&gmap, grad_pad, prows, 64))
    return cfail(2, "closure_wgrad64: tensor map encoding failed");
  static bool attr = false;
  const size_t smem = 1024 + kWStages * kWStageBytes + 128;
  if (!attr) {
    if (cudaFuncSetAttribute(k_wgrad64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return cfail(2, "closure_wgrad64: shared memory attribute");
    attr = true;
  }
  WgradArgs a;
  a.B = B; a.H = H; a.W = W; a.partials = partials; a.err = err;
  cudaStream_t st = (cudaStream_t)stream;
  k_wgrad64<<<nparts, kWThreads, smem, st>>>(amap, gmap, a);
  k_wgrad_reduce<<<(9 * 4096 + 255) / 256, 256, 0, st>>>(partials, nparts, dw);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cfail(2, std::string("closure_wgrad64 launch: ") + cudaGetErrorString(e));
  return 0;
}

}  // extern "C"
