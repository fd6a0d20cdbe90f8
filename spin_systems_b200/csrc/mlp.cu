// The echo surrogate's network on the device: a 6 -> 256 -> 256 -> 256 -> 128
// multilayer perceptron with GELU hidden activations, BF16 weights and
// activations, FP32 accumulation and FP32 master weights under Adam.
//
// Every matrix product -- the four forward layers, the backward data products
// and the weight gradients -- is one kernel, k_gemm:
//     C[M][N] = A[M][K] . B[N][K]^T,   A and B K-major BF16 in global memory.
// One CTA of four warps owns a 128-row x BN-column tile of C (BN = 32..256,
// picked per product so the grid covers the device).  Warp 0 stages 64-wide
// K slices of A and B into shared memory with TMA (128-byte swizzle) through
// a four-deep ring of mbarriers; warp 1 issues tcgen05.mma (kind::f16,
// BF16 x BF16 -> FP32, M = 128, N = BN, K = 16 per instruction) into a TMEM
// accumulator of BN columns and hands each stage back with tcgen05.commit;
// then all four warps read the accumulator with tcgen05.ld (TMEM lane = row
// of the tile) through a fused epilogue:
//   EPI_HIDDEN  z = acc + b, stored FP32; h = GELU(z) stored BF16 and, for
//               training, transposed (h^T is the K-major operand of the next
//               layer's weight gradient);
//   EPI_OUT     y = acc + b, FP32;
//   EPI_BACK    dz = acc * GELU'(z_below), stored FP32 (bias gradient),
//               BF16 and transposed BF16;
//   EPI_F32     plain FP32 store (weight gradients).
// The transposed BF16 tile is staged in the (by then idle) operand ring as
// [BN][128] and written back as 256-byte column runs with 16-byte stores.
// Waits on mbarriers are bounded by the global timer: a wait that runs out
// sets an error flag, the CTA still drains what it issued, frees its TMEM and
// returns, and the host reports SS_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace ss {
namespace mlp {

constexpr int kIn = 6;      // parameters per query
constexpr int kInPad = 64;  // input width as the first GEMM's K (one K slice)
constexpr int kHidden = 256;
constexpr int kOut = 128;   // echo points
constexpr int kLayers = 4;
constexpr int kRowsIn[kLayers] = {kInPad, kHidden, kHidden, kHidden};   // padded fan-in
constexpr int kTrueIn[kLayers] = {kIn, kHidden, kHidden, kHidden};
constexpr int kRowsOut[kLayers] = {kHidden, kHidden, kHidden, kOut};

constexpr int BM = 128;      // rows of C per CTA (tcgen05 M)
constexpr int BK = 64;       // K per stage: one 128-byte swizzle atom of BF16
constexpr int kStages = 4;
constexpr int kGemmThreads = 128;
constexpr uint32_t kABytes = BM * BK * 2;  // 16 KB
constexpr long long kWaitNs = 2000000000LL;  // 2 s bound on any mbarrier wait

constexpr int64_t param_count() {
  int64_t n = 0;
  for (int l = 0; l < kLayers; ++l) n += int64_t{kRowsOut[l]} * kTrueIn[l] + kRowsOut[l];
  return n;
}

enum Epi { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_BACK = 2, EPI_F32 = 3 };

struct GemmArgs {
  int M, N, K;
  int bn;                  // columns of C per CTA (gridDim.z = N / bn)
  const float* bias;       // HIDDEN, OUT: N
  float* out_f32;          // HIDDEN: z; OUT: y; BACK: dz; F32: C   ([M][N])
  __nv_bfloat16* out_bf;   // HIDDEN: GELU(z); BACK: dz             ([M][N])
  __nv_bfloat16* out_bt;   // the same, transposed ([N][M]); may be null
  const float* zin;        // BACK: pre-activation of the layer below ([M][N])
  int* flags;              // [0] set to 1 on a timed-out wait
  int splits;              // F32 only: K split over gridDim.y CTAs per row tile
  float* partial;          // splits > 1: [splits][M][N] FP32 slices, summed by k_splitk_sum
};

size_t gemm_smem(int bn) {
  return 1024 /* alignment slack */ + size_t{kStages} * (kABytes + size_t(bn) * BK * 2) + 256;
}
// The staged transposed tile ([bn][BM] BF16) fits in the B part of the
// operand ring it reuses ([kStages][bn][BK] BF16), whatever bn is.
static_assert(BM <= kStages * BK, "transposed staging outgrows the operand ring");

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// Waits for the phase of parity `parity` to complete; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long start = global_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - start > kWaitNs) return false;
  }
}

// One 2-D tile of a tensor map into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int k, int row) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(k), "r"(row)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile of 128-byte rows in the
// 128-byte swizzle: 8-row core groups 1024 bytes apart (stride byte offset),
// leading byte offset unused by this layout, descriptor version 1 (sm_100),
// layout type 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(1) << 16;
  d |= uint64_t(1024 >> 4) << 32;
  d |= uint64_t(1) << 46;
  d |= uint64_t(2) << 61;
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
// d/dz GELU = Phi(z) + z phi(z)
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// -------------------------------------------------------------- the GEMM
template <int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
           GemmArgs a) {
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte alignment in the shared window: the 128-byte swizzle pattern
  // of TMA and of the MMA descriptors is anchored there.
  uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int N = a.N;    // full width of C (row stride of the outputs)
  const int BN = a.bn;  // this CTA's columns: [n0, n0 + BN)
  const int n0 = blockIdx.z * BN;
  const uint32_t b_bytes = uint32_t(BN) * BK * 2;
  const uint32_t stage_bytes = kABytes + b_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * stage_bytes);
  uint64_t* full = bars;                  // TMA -> MMA
  uint64_t* empty = bars + kStages;       // MMA -> TMA
  uint64_t* done = bars + 2 * kStages;    // last MMA -> epilogue
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
  __shared__ int s_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ncols = BN <= 32 ? 32u : (BN <= 64 ? 64u : (BN <= 128 ? 128u : 256u));

  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(done), 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int m0 = blockIdx.x * BM;
  const int nk = a.K / BK / a.splits;      // k-tiles of this CTA's slice
  const int kbase = blockIdx.y * nk;       // its first k-tile

  if (warp == 0) {
    if (lane == 0) {
      // Producer: stage k-slices of A (128 rows) and B (BN rows).
      int issued = 0;
      bool ok = true;
      for (int kt = 0; kt < nk && ok; ++kt) {
        const int s = kt % kStages;
        if (kt >= kStages && !mbar_wait(smem_u32(&empty[s]), ((kt / kStages) & 1) ^ 1)) {
          ok = false;
          break;
        }
        uint8_t* sa = base + s * stage_bytes;
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, stage_bytes);
        tma_load_2d(smem_u32(sa), &map_a, fb, (kbase + kt) * BK, m0);
        tma_load_2d(smem_u32(sa + kABytes), &map_b, fb, (kbase + kt) * BK, n0);
        ++issued;
      }
      if (!ok) atomicExch(&s_fail, 1);
      // Drain: every copy issued has landed before the CTA may leave.
      for (int kt = std::max(0, issued - kStages); kt < issued; ++kt) {
        if (!mbar_wait(smem_u32(&full[kt % kStages]), (kt / kStages) & 1)) atomicExch(&s_fail, 1);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer.
      const uint32_t idesc = idesc_bf16(BM, BN);
      for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % kStages;
        if (!mbar_wait(smem_u32(&full[s]), (kt / kStages) & 1)) {
          atomicExch(&s_fail, 1);
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(base + s * stage_bytes);
        const uint32_t sb = sa + kABytes;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          umma_bf16(tmem, sw128_desc(sa + kk * 32), sw128_desc(sb + kk * 32), idesc,
                    (kt | kk) != 0 ? 1u : 0u);
        }
        umma_commit(smem_u32(&empty[s]));
      }
      umma_commit(smem_u32(done));  // also after a failure: nothing stays in flight
    }
    __syncwarp();
  }

  // Epilogue: every warp reads its 32 TMEM lanes (rows m0 + 32 warp + lane).
  if (!mbar_wait(smem_u32(done), 0)) atomicExch(&s_fail, 1);
  tc_fence_after();
  __syncthreads();
  const bool good = s_fail == 0;
  if (good) {
    const int row = m0 + warp * 32 + lane;
    const int M = a.M;
    // The operand ring is idle once `done` completed: every copy landed and
    // every MMA that read it finished.  It holds the transposed BF16 tile.
    __nv_bfloat16* stage_t = reinterpret_cast<__nv_bfloat16*>(base);
    for (int c0 = 0; c0 < BN; c0 += 16) {
      const int col = n0 + c0;
      float v[16];
      tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
      if (EPI == EPI_HIDDEN || EPI == EPI_OUT) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += a.bias[col + j];
      }
      if (EPI == EPI_BACK) {
        const float4* zp = reinterpret_cast<const float4*>(a.zin + size_t(row) * N + col);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 z = zp[q];
          v[4 * q + 0] *= gelu_grad(z.x);
          v[4 * q + 1] *= gelu_grad(z.y);
          v[4 * q + 2] *= gelu_grad(z.z);
          v[4 * q + 3] *= gelu_grad(z.w);
        }
      }
      float* out = (EPI == EPI_F32 && a.splits > 1)
                       ? a.partial + size_t(blockIdx.y) * size_t(M) * N
                       : a.out_f32;
      float4* fp = reinterpret_cast<float4*>(out + size_t(row) * N + col);
#pragma unroll
      for (int q = 0; q < 4; ++q) fp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      if (EPI == EPI_HIDDEN || EPI == EPI_BACK) {
        __nv_bfloat16 hb[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) hb[j] = __float2bfloat16_rn(EPI == EPI_HIDDEN ? gelu(v[j]) : v[j]);
        uint4* bp = reinterpret_cast<uint4*>(a.out_bf + size_t(row) * N + col);
        bp[0] = *reinterpret_cast<const uint4*>(&hb[0]);
        bp[1] = *reinterpret_cast<const uint4*>(&hb[8]);
        if (a.out_bt) {
          // A warp's 32 rows of one column are 64 contiguous bytes here.
#pragma unroll
          for (int j = 0; j < 16; ++j) stage_t[(c0 + j) * BM + warp * 32 + lane] = hb[j];
        }
      }
    }
    if ((EPI == EPI_HIDDEN || EPI == EPI_BACK) && a.out_bt) {
      __syncthreads();
      // Column c of the tile is rows m0 .. m0 + 127 of row n0 + c of C^T:
      // 16 stores of 16 bytes, consecutive threads on consecutive addresses.
      const uint4* src = reinterpret_cast<const uint4*>(stage_t);
      constexpr int kPerCol = BM / 8;
      for (int i = threadIdx.x; i < BN * kPerCol; i += kGemmThreads) {
        const int c = i / kPerCol, r8 = i % kPerCol;
        *reinterpret_cast<uint4*>(a.out_bt + size_t(n0 + c) * M + m0 + r8 * 8) = src[i];
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(a.flags, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
  }
}

// Sum of the split-K slices in slice order (deterministic): out = sum_s part[s].
__global__ void k_splitk_sum(const float4* __restrict__ part, int splits, size_t n4, float4* out) {
  const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n4) return;
  float4 acc = part[i];
  for (int s = 1; s < splits; ++s) {
    const float4 v = part[size_t(s) * n4 + i];
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
    acc.w += v.w;
  }
  out[i] = acc;
}

// ------------------------------------------------------- small kernels
// Rows per block of the batch kernels below: 256 threads, one warp per four
// rows for the 128-wide rows, one thread per 8-row x 1-column piece of a
// transposed row block.
constexpr int kRowBlock = 32;
constexpr int kRowThreads = 256;
constexpr int kTPitch = kRowBlock + 2;  // staged transposes: [column][row], padded

// Builds one batch: rows of the data set named by idx (or zero rows where
// idx < 0) as the padded BF16 input, its transpose, and the FP32 targets.
// With `cursor` (training graphs) the batch is rows cursor[0] * rows .. of idx.
// Every store is a whole 16-byte piece of a row (x, target) or of a
// transposed row (xt, through shared memory).
__global__ void __launch_bounds__(kRowThreads)
    k_gather(const float* __restrict__ data_x, const float* __restrict__ data_y,
             const int* __restrict__ idx_base, int rows, __nv_bfloat16* x, __nv_bfloat16* xt,
             float* target, const int* cursor) {
  __shared__ int s_row[kRowBlock];
  __shared__ __nv_bfloat16 s_in[kIn][kRowBlock];
  const int* idx = cursor ? idx_base + size_t(cursor[0]) * rows : idx_base;
  const int r0 = blockIdx.x * kRowBlock;
  const int t = threadIdx.x;
  if (t < kRowBlock) {
    const int i = idx[r0 + t];
    s_row[t] = i;
#pragma unroll
    for (int c = 0; c < kIn; ++c) {
      s_in[c][t] = __float2bfloat16_rn(i >= 0 ? data_x[size_t(i) * kIn + c] : 0.0f);
    }
  }
  __syncthreads();
  {
    // x: row t / 8, columns 8 (t % 8) .. + 7 (only the first piece is nonzero)
    const int r = t >> 3, q = t & 7;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * q + j;
      v[j] = c < kIn ? s_in[c][r] : __float2bfloat16_rn(0.0f);
    }
    *reinterpret_cast<uint4*>(x + size_t(r0 + r) * kInPad + 8 * q) = *reinterpret_cast<const uint4*>(v);
  }
  {
    // xt: column t / 4, rows 8 (t % 4) .. + 7 of the block
    const int c = t >> 2, part = t & 3;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = c < kIn ? s_in[c][8 * part + j] : __float2bfloat16_rn(0.0f);
    *reinterpret_cast<uint4*>(xt + size_t(c) * rows + r0 + 8 * part) = *reinterpret_cast<const uint4*>(v);
  }
  if (target) {
    // targets: warp w copies rows 4w .. 4w + 3, 16 bytes per lane per row
    const int w = t >> 5, lane = t & 31;
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = s_row[4 * w + k];
      v[k] = i >= 0 ? reinterpret_cast<const float4*>(data_y + size_t(i) * kOut)[lane]
                    : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      reinterpret_cast<float4*>(target + size_t(r0 + 4 * w + k) * kOut)[lane] = v[k];
    }
  }
}

// Mean-squared error over the first `valid` rows and the gradient of the
// output layer: g = 2 (y - t) / (valid * kOut), FP32, BF16 and transposed.
// Warp w of a block handles rows 4w .. 4w + 3 of its 32, lane l columns
// 4l .. 4l + 3 (16-byte loads and stores along the rows); the transposed
// BF16 block is staged in shared memory and written as 16-byte pieces.
// The block's squared error is summed in a fixed order (deterministic).
__global__ void __launch_bounds__(kRowThreads)
    k_loss(const float* __restrict__ y, const float* __restrict__ t, int rows, int valid, float* g,
           __nv_bfloat16* dz, __nv_bfloat16* dzt, double* partial) {
  __shared__ __nv_bfloat16 s_t[kOut][kTPitch];
  __shared__ double red[kRowThreads / 32];
  const int r0 = blockIdx.x * kRowBlock;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float scale = 2.0f / (float(valid) * float(kOut));
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rl = 4 * w + k, r = r0 + rl;
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (r < valid) {
      const float4 a = reinterpret_cast<const float4*>(y + size_t(r) * kOut)[lane];
      const float4 b = reinterpret_cast<const float4*>(t + size_t(r) * kOut)[lane];
      d[0] = a.x - b.x;
      d[1] = a.y - b.y;
      d[2] = a.z - b.z;
      d[3] = a.w - b.w;
    }
    __align__(8) __nv_bfloat16 hb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc += double(d[j]) * double(d[j]);
      d[j] *= scale;
      hb[j] = __float2bfloat16_rn(d[j]);
      s_t[4 * lane + j][rl] = hb[j];
    }
    reinterpret_cast<float4*>(g + size_t(r) * kOut)[lane] = make_float4(d[0], d[1], d[2], d[3]);
    *reinterpret_cast<uint2*>(dz + size_t(r) * kOut + 4 * lane) = *reinterpret_cast<const uint2*>(hb);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (lane == 0) red[w] = acc;
  __syncthreads();
  // dzt: column c, rows 8 part .. + 7 of the block; two pieces per thread
#pragma unroll
  for (int i = threadIdx.x; i < kOut * 4; i += kRowThreads) {
    const int c = i >> 2, part = i & 3;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = s_t[c][8 * part + j];
    *reinterpret_cast<uint4*>(dzt + size_t(c) * rows + r0 + 8 * part) = *reinterpret_cast<const uint4*>(v);
  }
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int k = 0; k < kRowThreads / 32; ++k) sum += red[k];
    partial[blockIdx.x] = sum;
  }
}

// loss[slot] = sum of the block partials / (valid * kOut), in block order;
// with `cursor` (training graphs) the slot is the step index cursor[1].
__global__ void k_loss_total(const double* partial, int nblocks, int valid, double* loss, int slot,
                             const int* cursor) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b];
    loss[cursor ? cursor[1] : slot] = s / (double(valid) * double(kOut));
  }
}

// The training graph's step counter: batch position in the epoch, step index.
__global__ void k_advance(int* cursor, int per_epoch) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    cursor[0] = (cursor[0] + 1) % per_epoch;
    cursor[1] += 1;
  }
}

// Column sums of g[rows][N] (the bias gradient) in two deterministic stages:
// blocks of 32 columns x 256 rows write partial sums, then one pass adds the
// partials in row-block order.
constexpr int kColRows = 256;
__global__ void k_colsum_part(const float* __restrict__ g, int rows, int N, float* part) {
  __shared__ float red[8][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  const int r0 = blockIdx.y * kColRows;
  float s = 0.0f;
  if (c < N) {
#pragma unroll 8
    for (int i = 0; i < kColRows / 8; ++i) {
      const int r = r0 + threadIdx.y + 8 * i;
      if (r < rows) s += g[size_t(r) * N + c];
    }
  }
  red[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < N) {
    float t = 0.0f;
    for (int y = 0; y < 8; ++y) t += red[y][threadIdx.x];
    part[size_t(blockIdx.y) * N + c] = t;
  }
}

__global__ void k_colsum_fin(const float* __restrict__ part, int nblocks, int N, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.0f;
  for (int b = 0; b < nblocks; ++b) s += part[size_t(b) * N + c];
  out[c] = s;
}

// One parameter tensor for the Adam step.
struct Seg {
  long long off;          // first element in the flat parameter vector
  int rows, cols, pitch;  // weight: rows x cols (cols = true fan-in), grad pitch = padded fan-in
  const float* grad;      // gradient ([rows][pitch] for weights, [rows] for biases)
  __nv_bfloat16* w;       // BF16 copy [rows][pitch] (null for biases)
  __nv_bfloat16* wt;      // BF16 transpose [pitch][rows]
};
struct Segs {
  Seg s[2 * kLayers];
};

// Adam on the FP32 master parameters (update = 1), then the BF16 copies the
// GEMMs read.  update = 0 only refreshes the copies.
// With `lr_steps` (training graphs) the step's learning rate is
// lr_steps[cursor[1]].
__global__ void k_adam(Segs segs, float* p, float* m, float* v, long long total, float lr_host,
                       float b1, float b2, float eps, int update, const float* lr_steps,
                       const int* cursor) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= total) return;
  const float lr_t = lr_steps ? lr_steps[cursor[1]] : lr_host;
  int k = 0;
  while (k + 1 < 2 * kLayers && i >= segs.s[k + 1].off) ++k;
  const Seg& sg = segs.s[k];
  const long long local = i - sg.off;
  float w = p[i];
  if (sg.w) {
    const int r = static_cast<int>(local / sg.cols), c = static_cast<int>(local % sg.cols);
    if (update) {
      const float g = sg.grad[size_t(r) * sg.pitch + c];
      const float mi = b1 * m[i] + (1.0f - b1) * g;
      const float vi = b2 * v[i] + (1.0f - b2) * g * g;
      m[i] = mi;
      v[i] = vi;
      w -= lr_t * mi / (sqrtf(vi) + eps);
      p[i] = w;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(w);
    sg.w[size_t(r) * sg.pitch + c] = b;
    sg.wt[size_t(c) * sg.rows + r] = b;
  } else if (update) {
    const float g = sg.grad[local];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    p[i] = w - lr_t * mi / (sqrtf(vi) + eps);
  }
}

// --------------------------------------------------------- tensor maps
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    SS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    require(p != nullptr && q == cudaDriverEntryPointSuccess, SS_ERR_CUDA,
            "cuTensorMapEncodeTiled is not available from the driver");
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// Map of a row-major BF16 matrix [rows][cols] (cols = K, a multiple of 64)
// read as boxes of 64 K-elements x box_rows rows in the 128-byte swizzle.
CUtensorMap make_map(const __nv_bfloat16* ptr, int rows, int cols, int box_rows) {
  require(cols % BK == 0 && rows % 8 == 0 && box_rows <= 256 && rows >= box_rows, SS_ERR_RUNTIME,
          "tensor map shape");
  require((reinterpret_cast<uintptr_t>(ptr) & 15u) == 0, SS_ERR_RUNTIME, "tensor map alignment");
  CUtensorMap m;
  const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(cols) * 2};
  const cuuint32_t box[2] = {BK, cuuint32_t(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                 const_cast<__nv_bfloat16*>(ptr), dims, strides, box, elem,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  require(r == CUDA_SUCCESS, SS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return m;
}

// One prepared product: operands' maps and the epilogue's pointers.
struct Gemm {
  CUtensorMap ma, mb;
  GemmArgs args;
  int epi;
};

// splitmix64, for weight initialisation and batch shuffles.
inline uint64_t mix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline double unit(uint64_t& s) { return double(mix64(s) >> 11) * 0x1.0p-53; }

}  // namespace mlp
}  // namespace ss

using namespace ss;
using namespace ss::mlp;

struct ss_mlp {
  ss_engine* engine = nullptr;
  int batch = 0;       // rows per device pass (multiple of 128)
  int64_t steps = 0;   // Adam steps taken
  // parameters, FP32 master copy in the flat ABI order, and Adam moments
  float* p = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* gw[kLayers] = {};  // weight gradients [out][padded in]
  float* gb[kLayers] = {};  // bias gradients [out]
  __nv_bfloat16* w[kLayers] = {};   // [out][padded in]
  __nv_bfloat16* wt[kLayers] = {};  // [padded in][out]
  long long w_off[kLayers] = {}, b_off[kLayers] = {};
  // activations of one batch
  __nv_bfloat16 *x = nullptr, *xt = nullptr;
  float* z[3] = {};
  __nv_bfloat16* h[3] = {};
  __nv_bfloat16* ht[3] = {};
  float* y = nullptr;
  float* target = nullptr;
  float* g = nullptr;                       // FP32 gradient of the current layer
  __nv_bfloat16* dz[2] = {};                // ping-pong [batch][256]
  __nv_bfloat16* dzt[2] = {};               // [256][batch]
  double* loss_part = nullptr;
  float* col_part = nullptr;                // column-sum partials
  float* splitk = nullptr;                  // split-K slices of the weight gradients
  int* cursor = nullptr;                    // training graph: epoch position, step index
  float* lr_steps = nullptr;                // training graph: learning rate per step
  int64_t lr_cap = 0;
  double* losses = nullptr;                 // per-step losses of the last train call
  int64_t losses_cap = 0;
  int* idx = nullptr;                       // batch rows (data-set indices)
  int64_t idx_cap = 0;
  // training set
  float* data_x = nullptr;
  float* data_y = nullptr;
  int64_t data_n = 0;
  // prepared products
  Gemm fwd[kLayers];
  Gemm bwd_w[kLayers];   // weight gradient of layer l
  Gemm bwd_x[kLayers];   // data gradient into layer l - 1 (l >= 1)
  Segs segs;
};

namespace ss {
namespace mlp {
namespace {

template <typename T>
void dalloc(T** p, size_t n) {
  SS_CUDA(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * std::max<size_t>(n, 1)));
  SS_CUDA(cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(n, 1)));
}

void launch_gemm(ss_engine* e, const Gemm& gm) {
  const GemmArgs& a = gm.args;
  const dim3 grid(a.M / BM, a.splits, a.N / a.bn);
  const size_t smem = gemm_smem(a.bn);
  switch (gm.epi) {
    case EPI_HIDDEN: launch(e, k_gemm<EPI_HIDDEN>, grid, kGemmThreads, smem, gm.ma, gm.mb, a); break;
    case EPI_OUT: launch(e, k_gemm<EPI_OUT>, grid, kGemmThreads, smem, gm.ma, gm.mb, a); break;
    case EPI_BACK: launch(e, k_gemm<EPI_BACK>, grid, kGemmThreads, smem, gm.ma, gm.mb, a); break;
    default: launch(e, k_gemm<EPI_F32>, grid, kGemmThreads, smem, gm.ma, gm.mb, a); break;
  }
  if (a.splits > 1) {
    const size_t n4 = size_t(a.M) * a.N / 4;
    launch(e, k_splitk_sum, dim3(static_cast<unsigned>((n4 + 255) / 256)), 256, 0,
           reinterpret_cast<const float4*>(a.partial), a.splits, n4,
           reinterpret_cast<float4*>(a.out_f32));
  }
}

void run_gemm(ss_mlp* n, const Gemm& gm) { launch_gemm(n->engine, gm); }

// K slices for a weight-gradient product (K = the batch, long; M = a layer
// width, one or two row tiles): enough CTAs to spread over the device with
// at least four k-tiles each, a power of two dividing the k-tile count.
int splitk_for(int M, int K) {
  const int nk = K / BK;
  const int want = std::max(1, 64 / std::max(1, M / BM));
  int s = 1;
  while (s * 2 <= want && nk % (s * 2) == 0 && nk / (s * 2) >= 4) s *= 2;
  return s;
}

// Columns of C per CTA: halved from the full width (down to 32, and only
// while it stays a multiple of 16 dividing the width) while the
// grid of row tiles x K slices x column tiles has fewer CTAs than the device
// has SMs.  Short-K products are bound by their epilogues, which then run on
// more SMs with fewer columns each.
int column_tile(int M, int N, int splits) {
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) {
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  int bn = N;
  while (bn > 32 && bn % 32 == 0 && (M / BM) * splits * (N / bn) < sms) bn /= 2;
  return bn;
}

Gemm make_gemm(int epi, const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K,
               int* flags, int splits = 1) {
  require(M % BM == 0 && K % BK == 0 && N % 16 == 0 && N >= 16 && N <= 256, SS_ERR_RUNTIME,
          "GEMM shape outside the tcgen05 tiling");
  Gemm g{};
  g.args.M = M;
  g.args.N = N;
  g.args.K = K;
  g.args.flags = flags;
  g.args.splits = splits;
  g.args.bn = column_tile(M, N, splits);
  g.ma = make_map(A, M, K, BM);
  g.mb = make_map(B, N, K, g.args.bn);
  g.epi = epi;
  return g;
}

void set_smem_attrs() {
  static bool done = [] {
    const int bytes = static_cast<int>(gemm_smem(256));
    SS_CUDA(cudaFuncSetAttribute(k_gemm<EPI_HIDDEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SS_CUDA(cudaFuncSetAttribute(k_gemm<EPI_OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SS_CUDA(cudaFuncSetAttribute(k_gemm<EPI_BACK>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SS_CUDA(cudaFuncSetAttribute(k_gemm<EPI_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return true;
  }();
  (void)done;
}

void build(ss_mlp* n) {
  const int B = n->batch;
  int* flags = n->engine->dev_flags + 8;
  // parameter segments in the flat ABI order: W0 b0 W1 b1 W2 b2 W3 b3
  long long off = 0;
  for (int l = 0; l < kLayers; ++l) {
    n->w_off[l] = off;
    off += static_cast<long long>(kRowsOut[l]) * kTrueIn[l];
    n->b_off[l] = off;
    off += kRowsOut[l];
  }
  const size_t P = static_cast<size_t>(param_count());
  dalloc(&n->p, P);
  dalloc(&n->m, P);
  dalloc(&n->v, P);
  for (int l = 0; l < kLayers; ++l) {
    dalloc(&n->gw[l], size_t(kRowsOut[l]) * kRowsIn[l]);
    dalloc(&n->gb[l], size_t(kRowsOut[l]));
    dalloc(&n->w[l], size_t(kRowsOut[l]) * kRowsIn[l]);
    dalloc(&n->wt[l], size_t(kRowsOut[l]) * kRowsIn[l]);
    n->segs.s[2 * l] = Seg{n->w_off[l], kRowsOut[l], kTrueIn[l], kRowsIn[l], n->gw[l], n->w[l], n->wt[l]};
    n->segs.s[2 * l + 1] = Seg{n->b_off[l], kRowsOut[l], 1, 1, n->gb[l], nullptr, nullptr};
  }
  dalloc(&n->x, size_t(B) * kInPad);
  dalloc(&n->xt, size_t(B) * kInPad);
  for (int l = 0; l < 3; ++l) {
    dalloc(&n->z[l], size_t(B) * kHidden);
    dalloc(&n->h[l], size_t(B) * kHidden);
    dalloc(&n->ht[l], size_t(B) * kHidden);
  }
  dalloc(&n->y, size_t(B) * kOut);
  dalloc(&n->target, size_t(B) * kOut);
  dalloc(&n->g, size_t(B) * kHidden);
  for (int i = 0; i < 2; ++i) {
    dalloc(&n->dz[i], size_t(B) * kHidden);
    dalloc(&n->dzt[i], size_t(B) * kHidden);
  }
  dalloc(&n->loss_part, size_t(B / kRowBlock));
  dalloc(&n->col_part, size_t(B / kColRows + 1) * kHidden);
  n->idx_cap = B;
  dalloc(&n->idx, size_t(B));

  set_smem_attrs();
  // forward: layer l reads x or h[l-1] and the BF16 weights [out][in]
  for (int l = 0; l < kLayers; ++l) {
    const __nv_bfloat16* A = l == 0 ? n->x : n->h[l - 1];
    Gemm g = make_gemm(l < 3 ? EPI_HIDDEN : EPI_OUT, A, n->w[l], B, kRowsOut[l], kRowsIn[l], flags);
    g.args.bias = n->p + n->b_off[l];
    if (l < 3) {
      g.args.out_f32 = n->z[l];
      g.args.out_bf = n->h[l];
      g.args.out_bt = n->ht[l];
    } else {
      g.args.out_f32 = n->y;
    }
    n->fwd[l] = g;
  }
  // backward: dz of layer l lives in dz[(3 - l) & 1] (layer 3 in slot 0)
  for (int l = kLayers - 1; l >= 0; --l) {
    const int slot = (3 - l) & 1;
    const __nv_bfloat16* inT = l == 0 ? n->xt : n->ht[l - 1];  // [in][B]
    Gemm gw = make_gemm(EPI_F32, n->dzt[slot], inT, kRowsOut[l], kRowsIn[l], B, flags,
                        splitk_for(kRowsOut[l], B));
    gw.args.out_f32 = n->gw[l];
    n->bwd_w[l] = gw;
    if (l >= 1) {
      Gemm gx = make_gemm(EPI_BACK, n->dz[slot], n->wt[l], B, kRowsIn[l], kRowsOut[l], flags);
      gx.args.zin = n->z[l - 1];
      gx.args.out_f32 = n->g;
      gx.args.out_bf = n->dz[slot ^ 1];
      gx.args.out_bt = n->dzt[slot ^ 1];
      n->bwd_x[l] = gx;
    }
  }
  // one workspace for the split-K slices, shared by the (serial) products
  size_t ws = 0;
  for (int l = 0; l < kLayers; ++l) {
    const GemmArgs& a = n->bwd_w[l].args;
    if (a.splits > 1) ws = std::max(ws, size_t(a.splits) * a.M * a.N);
  }
  if (ws > 0) dalloc(&n->splitk, ws);
  for (int l = 0; l < kLayers; ++l) n->bwd_w[l].args.partial = n->splitk;
}

void refresh_copies(ss_mlp* n, float lr_t, int update, const float* lr_steps = nullptr,
                    const int* cursor = nullptr) {
  const long long total = param_count();
  launch(n->engine, k_adam, dim3(static_cast<unsigned>((total + 255) / 256)), 256, 0, n->segs,
         n->p, n->m, n->v, total, lr_t, 0.9f, 0.999f, 1e-8f, update, lr_steps, cursor);
}

void forward(ss_mlp* n, bool keep_transposes) {
  for (int l = 0; l < kLayers; ++l) {
    Gemm g = n->fwd[l];
    if (!keep_transposes) g.args.out_bt = nullptr;
    run_gemm(n, g);
  }
}

// Bias gradient: column sums of the FP32 layer gradient g[batch][N].
void colsum(ss_mlp* n, int N, float* out) {
  const int B = n->batch;
  const int nb = (B + kColRows - 1) / kColRows;
  launch(n->engine, k_colsum_part, dim3((N + 31) / 32, nb), dim3(32, 8), 0, n->g, B, N,
         n->col_part);
  launch(n->engine, k_colsum_fin, dim3((N + 127) / 128), 128, 0, n->col_part, nb, N, out);
}

// Backward pass of the batch in x / target (loss over the first `valid`
// rows); writes gw, gb and the loss into losses[slot].
void backward(ss_mlp* n, int valid, double* loss, int slot, const int* cursor = nullptr) {
  ss_engine* e = n->engine;
  const int B = n->batch;
  const int nb = B / kRowBlock;
  launch(e, k_loss, dim3(nb), kRowThreads, 0, n->y, n->target, B, valid, n->g, n->dz[0],
         n->dzt[0], n->loss_part);
  launch(e, k_loss_total, dim3(1), 32, 0, n->loss_part, nb, valid, loss, slot, cursor);
  colsum(n, kOut, n->gb[3]);
  for (int l = kLayers - 1; l >= 0; --l) {
    run_gemm(n, n->bwd_w[l]);
    if (l >= 1) {
      run_gemm(n, n->bwd_x[l]);
      colsum(n, kRowsIn[l], n->gb[l - 1]);
    }
  }
}

void gather(ss_mlp* n, const float* dx, const float* dy, const int* idx,
            const int* cursor = nullptr) {
  const int B = n->batch;
  launch(n->engine, k_gather, dim3(B / kRowBlock), kRowThreads, 0, dx, dy, idx, B, n->x,
         n->xt, dy ? n->target : nullptr, cursor);
}

void check_timeout(ss_mlp* n) {
  ss_engine* e = n->engine;
  int flag = 0;
  SS_CUDA(cudaMemcpyAsync(&flag, e->dev_flags + 8, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  sync(e);
  if (flag) {
    SS_CUDA(cudaMemsetAsync(e->dev_flags + 8, 0, sizeof(int), e->stream));
    sync(e);
    fail(SS_ERR_TIMEOUT, "a tensor-core GEMM wait timed out");
  }
}

void check_mlp(const ss_mlp* n) {
  require(n != nullptr && n->engine != nullptr, SS_ERR_INVALID_ARGUMENT, "null network");
}

}  // namespace
}  // namespace mlp
}  // namespace ss

extern "C" {

int64_t ss_mlp_param_count(void) { return param_count(); }

int ss_mlp_create(ss_engine* e, int batch, uint64_t seed, ss_mlp** out) {
  return guarded([&] {
    require(e != nullptr && out != nullptr, SS_ERR_INVALID_ARGUMENT, "null argument");
    require(batch >= BM && batch % BM == 0 && batch <= (1 << 16), SS_ERR_INVALID_ARGUMENT,
            "batch must be a multiple of 128 in [128, 65536]");
    SS_CUDA(cudaSetDevice(e->device));
    auto* n = new ss_mlp;
    n->engine = e;
    n->batch = batch;
    try {
      build(n);
      // He-uniform weights for the GELU layers, a smaller scale for the
      // linear output layer, zero biases.
      std::vector<float> p(static_cast<size_t>(param_count()), 0.0f);
      uint64_t s = seed ^ 0x6A09E667F3BCC909ull;
      for (int l = 0; l < kLayers; ++l) {
        const double a = (l < 3 ? std::sqrt(6.0) : std::sqrt(3.0)) / std::sqrt(double(kTrueIn[l]));
        const size_t cnt = size_t(kRowsOut[l]) * kTrueIn[l];
        for (size_t i = 0; i < cnt; ++i) p[n->w_off[l] + i] = float((2.0 * unit(s) - 1.0) * a);
      }
      SS_CUDA(cudaMemcpyAsync(n->p, p.data(), sizeof(float) * p.size(), cudaMemcpyHostToDevice, e->stream));
      refresh_copies(n, 0.0f, 0);
      sync(e);
    } catch (...) {
      ss_mlp_destroy(n);
      throw;
    }
    *out = n;
  });
}

int ss_mlp_destroy(ss_mlp* n) {
  return guarded([&] {
    if (n == nullptr) return;
    if (n->engine && n->engine->stream) cudaStreamSynchronize(n->engine->stream);
    void* ptrs[] = {n->p, n->m, n->v, n->x, n->xt, n->y, n->target, n->g, n->loss_part,
                    n->col_part, n->splitk, n->cursor, n->lr_steps, n->losses, n->idx,
                    n->data_x, n->data_y};
    for (void* q : ptrs) cudaFree(q);
    for (int l = 0; l < kLayers; ++l) {
      cudaFree(n->gw[l]);
      cudaFree(n->gb[l]);
      cudaFree(n->w[l]);
      cudaFree(n->wt[l]);
    }
    for (int l = 0; l < 3; ++l) {
      cudaFree(n->z[l]);
      cudaFree(n->h[l]);
      cudaFree(n->ht[l]);
    }
    for (int i = 0; i < 2; ++i) {
      cudaFree(n->dz[i]);
      cudaFree(n->dzt[i]);
    }
    delete n;
  });
}

int ss_mlp_get_params(const ss_mlp* n, float* out) {
  return guarded([&] {
    check_mlp(n);
    require(out != nullptr, SS_ERR_INVALID_ARGUMENT, "null output");
    SS_CUDA(cudaMemcpyAsync(out, n->p, sizeof(float) * param_count(), cudaMemcpyDeviceToHost,
                            n->engine->stream));
    sync(n->engine);
  });
}

int ss_mlp_set_params(ss_mlp* n, const float* in) {
  return guarded([&] {
    check_mlp(n);
    require(in != nullptr, SS_ERR_INVALID_ARGUMENT, "null input");
    ss_engine* e = n->engine;
    const size_t P = static_cast<size_t>(param_count());
    SS_CUDA(cudaMemcpyAsync(n->p, in, sizeof(float) * P, cudaMemcpyHostToDevice, e->stream));
    SS_CUDA(cudaMemsetAsync(n->m, 0, sizeof(float) * P, e->stream));
    SS_CUDA(cudaMemsetAsync(n->v, 0, sizeof(float) * P, e->stream));
    n->steps = 0;
    refresh_copies(n, 0.0f, 0);
    sync(e);
  });
}

int ss_mlp_forward(ss_mlp* n, const float* x, int64_t rows, float* y) {
  return guarded([&] {
    check_mlp(n);
    require(rows >= 0 && (rows == 0 || (x != nullptr && y != nullptr)), SS_ERR_INVALID_ARGUMENT,
            "bad forward buffers");
    ss_engine* e = n->engine;
    const int B = n->batch;
    float* dx = nullptr;
    SS_CUDA(cudaMalloc(&dx, sizeof(float) * size_t(B) * kIn));
    std::vector<int> idx(B);
    try {
      for (int64_t at = 0; at < rows; at += B) {
        const int cnt = static_cast<int>(std::min<int64_t>(B, rows - at));
        for (int r = 0; r < B; ++r) idx[r] = r < cnt ? r : -1;
        SS_CUDA(cudaMemcpyAsync(dx, x + at * kIn, sizeof(float) * cnt * kIn, cudaMemcpyHostToDevice, e->stream));
        SS_CUDA(cudaMemcpyAsync(n->idx, idx.data(), sizeof(int) * B, cudaMemcpyHostToDevice, e->stream));
        gather(n, dx, nullptr, n->idx);
        forward(n, false);
        SS_CUDA(cudaMemcpyAsync(y + at * kOut, n->y, sizeof(float) * cnt * kOut, cudaMemcpyDeviceToHost, e->stream));
        sync(e);
      }
      check_timeout(n);
    } catch (...) {
      cudaFree(dx);
      throw;
    }
    cudaFree(dx);
  });
}

int ss_mlp_gradients(ss_mlp* n, const float* x, const float* target, int64_t rows, float* grads,
                     double* loss) {
  return guarded([&] {
    check_mlp(n);
    require(x != nullptr && target != nullptr && grads != nullptr, SS_ERR_INVALID_ARGUMENT,
            "null buffer");
    require(rows >= 1 && rows <= n->batch, SS_ERR_INVALID_ARGUMENT, "rows must be in [1, batch]");
    ss_engine* e = n->engine;
    const int B = n->batch;
    float *dx = nullptr, *dy = nullptr;
    double* dl = nullptr;
    SS_CUDA(cudaMalloc(&dx, sizeof(float) * size_t(rows) * kIn));
    SS_CUDA(cudaMalloc(&dy, sizeof(float) * size_t(rows) * kOut));
    SS_CUDA(cudaMalloc(&dl, sizeof(double)));
    std::vector<int> idx(B);
    for (int r = 0; r < B; ++r) idx[r] = r < rows ? r : -1;
    try {
      SS_CUDA(cudaMemcpyAsync(dx, x, sizeof(float) * rows * kIn, cudaMemcpyHostToDevice, e->stream));
      SS_CUDA(cudaMemcpyAsync(dy, target, sizeof(float) * rows * kOut, cudaMemcpyHostToDevice, e->stream));
      SS_CUDA(cudaMemcpyAsync(n->idx, idx.data(), sizeof(int) * B, cudaMemcpyHostToDevice, e->stream));
      gather(n, dx, dy, n->idx);
      forward(n, true);
      backward(n, static_cast<int>(rows), dl, 0);
      std::vector<float> gw, gb;
      double lv = 0.0;
      for (int l = 0; l < kLayers; ++l) {
        gw.resize(size_t(kRowsOut[l]) * kRowsIn[l]);
        gb.resize(size_t(kRowsOut[l]));
        SS_CUDA(cudaMemcpyAsync(gw.data(), n->gw[l], sizeof(float) * gw.size(), cudaMemcpyDeviceToHost, e->stream));
        SS_CUDA(cudaMemcpyAsync(gb.data(), n->gb[l], sizeof(float) * gb.size(), cudaMemcpyDeviceToHost, e->stream));
        if (l == 0) SS_CUDA(cudaMemcpyAsync(&lv, dl, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        sync(e);
        for (int r = 0; r < kRowsOut[l]; ++r) {
          for (int c = 0; c < kTrueIn[l]; ++c) {
            grads[n->w_off[l] + int64_t(r) * kTrueIn[l] + c] = gw[size_t(r) * kRowsIn[l] + c];
          }
          grads[n->b_off[l] + r] = gb[r];
        }
      }
      if (loss) *loss = lv;
      check_timeout(n);
    } catch (...) {
      cudaFree(dx);
      cudaFree(dy);
      cudaFree(dl);
      throw;
    }
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dl);
  });
}

int ss_mlp_set_data(ss_mlp* n, const float* x, const float* y, int64_t rows) {
  return guarded([&] {
    check_mlp(n);
    require(x != nullptr && y != nullptr && rows >= n->batch, SS_ERR_INVALID_ARGUMENT,
            "the training set needs at least one full batch of rows");
    require(rows < (int64_t{1} << 31), SS_ERR_INVALID_ARGUMENT, "training set too large");
    ss_engine* e = n->engine;
    sync(e);
    cudaFree(n->data_x);
    cudaFree(n->data_y);
    n->data_x = n->data_y = nullptr;
    n->data_n = 0;
    SS_CUDA(cudaMalloc(&n->data_x, sizeof(float) * size_t(rows) * kIn));
    SS_CUDA(cudaMalloc(&n->data_y, sizeof(float) * size_t(rows) * kOut));
    SS_CUDA(cudaMemcpyAsync(n->data_x, x, sizeof(float) * size_t(rows) * kIn, cudaMemcpyHostToDevice, e->stream));
    SS_CUDA(cudaMemcpyAsync(n->data_y, y, sizeof(float) * size_t(rows) * kOut, cudaMemcpyHostToDevice, e->stream));
    if (n->idx_cap < rows) {
      cudaFree(n->idx);
      n->idx = nullptr;
      SS_CUDA(cudaMalloc(&n->idx, sizeof(int) * size_t(rows)));
      n->idx_cap = rows;
    }
    sync(e);
    n->data_n = rows;
  });
}

int ss_mlp_train(ss_mlp* n, int64_t steps, float lr_start, float lr_end, uint64_t seed,
                 double* losses) {
  return guarded([&] {
    TraceRange trace("ss_mlp_train");
    check_mlp(n);
    require(n->data_n >= n->batch, SS_ERR_INVALID_ARGUMENT, "no training set (ss_mlp_set_data)");
    require(steps >= 0, SS_ERR_INVALID_ARGUMENT, "negative step count");
    require(lr_start >= 0.0f && lr_end >= 0.0f, SS_ERR_INVALID_ARGUMENT, "negative learning rate");
    ss_engine* e = n->engine;
    const int B = n->batch;
    if (n->losses_cap < steps) {
      cudaFree(n->losses);
      n->losses = nullptr;
      SS_CUDA(cudaMalloc(&n->losses, sizeof(double) * size_t(std::max<int64_t>(steps, 1))));
      n->losses_cap = steps;
    }
    const int64_t per_epoch = n->data_n / B;
    require(per_epoch < (int64_t{1} << 30) && steps < (int64_t{1} << 31), SS_ERR_INVALID_ARGUMENT,
            "too many steps");
    // Learning rate per step (cosine from lr_start to lr_end) with Adam's bias
    // correction folded in, for the graph to read by step index.
    std::vector<float> lr(static_cast<size_t>(std::max<int64_t>(steps, 1)));
    for (int64_t t = 0; t < steps; ++t) {
      const double frac = steps > 1 ? double(t) / double(steps - 1) : 0.0;
      const double base = lr_end + 0.5 * (lr_start - lr_end) * (1.0 + std::cos(3.14159265358979323846 * frac));
      const double k = double(n->steps + t + 1);
      const double c1 = 1.0 - std::pow(0.9, k), c2 = 1.0 - std::pow(0.999, k);
      lr[t] = static_cast<float>(base * std::sqrt(c2) / c1);
    }
    if (n->lr_cap < steps) {
      cudaFree(n->lr_steps);
      n->lr_steps = nullptr;
      SS_CUDA(cudaMalloc(&n->lr_steps, sizeof(float) * lr.size()));
      n->lr_cap = steps;
    }
    if (!n->cursor) SS_CUDA(cudaMalloc(&n->cursor, 2 * sizeof(int)));
    SS_CUDA(cudaMemcpyAsync(n->lr_steps, lr.data(), sizeof(float) * lr.size(), cudaMemcpyHostToDevice, e->stream));
    SS_CUDA(cudaMemsetAsync(n->cursor, 0, 2 * sizeof(int), e->stream));
    // One step -- gather, forward, loss, backward, Adam, advance -- captured
    // once as a CUDA graph and replayed: the step's ~25 launches would
    // otherwise bound it.  What changes per step (batch position, loss slot,
    // learning rate) is read from device memory by step index.
    cudaGraphExec_t exec = nullptr;
    if (steps > 0) {
      cudaGraph_t graph = nullptr;
      SS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      try {
        gather(n, n->data_x, n->data_y, n->idx, n->cursor);
        forward(n, true);
        backward(n, B, n->losses, 0, n->cursor);
        refresh_copies(n, 0.0f, 1, n->lr_steps, n->cursor);
        launch(e, k_advance, dim3(1), 32, 0, n->cursor, static_cast<int>(per_epoch));
      } catch (...) {
        cudaStreamEndCapture(e->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      SS_CUDA(cudaStreamEndCapture(e->stream, &graph));
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      SS_CUDA(ie);
    }
    std::vector<int> perm(static_cast<size_t>(n->data_n));
    uint64_t s = seed ^ 0xBB67AE8584CAA73Bull;
    try {
      for (int64_t t = 0; t < steps; ++t) {
        if (t % per_epoch == 0) {
          for (int64_t i = 0; i < n->data_n; ++i) perm[i] = static_cast<int>(i);
          for (int64_t i = n->data_n - 1; i > 0; --i) {
            const int64_t j = static_cast<int64_t>(mix64(s) % uint64_t(i + 1));
            std::swap(perm[i], perm[j]);
          }
          SS_CUDA(cudaMemcpyAsync(n->idx, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, e->stream));
          sync(e);  // perm is reused on the host
        }
        SS_CUDA(cudaGraphLaunch(exec, e->stream));
      }
    } catch (...) {
      if (exec) cudaGraphExecDestroy(exec);
      throw;
    }
    if (exec) {
      sync(e);
      cudaGraphExecDestroy(exec);
    }
    n->steps += steps;
    if (losses && steps > 0) {
      SS_CUDA(cudaMemcpyAsync(losses, n->losses, sizeof(double) * size_t(steps), cudaMemcpyDeviceToHost, e->stream));
    }
    sync(e);
    check_timeout(n);
  });
}

int ss_mlp_gemm_test(ss_engine* e, const uint16_t* a, const uint16_t* b, int M, int N, int K,
                     float* c) {
  return guarded([&] {
    require(e != nullptr && a != nullptr && b != nullptr && c != nullptr, SS_ERR_INVALID_ARGUMENT,
            "null argument");
    require(M >= BM && M % BM == 0 && K >= BK && K % BK == 0 && N % 16 == 0 && N >= 16 && N <= 256,
            SS_ERR_INVALID_ARGUMENT, "shape outside the tcgen05 tiling (M%128, K%64, N%16<=256)");
    SS_CUDA(cudaSetDevice(e->device));
    set_smem_attrs();
    __nv_bfloat16 *da = nullptr, *db = nullptr;
    float *dc = nullptr, *dp = nullptr;
    auto cleanup = [&] {
      cudaFree(da);
      cudaFree(db);
      cudaFree(dc);
      cudaFree(dp);
    };
    try {
      SS_CUDA(cudaMalloc(&da, sizeof(uint16_t) * size_t(M) * K));
      SS_CUDA(cudaMalloc(&db, sizeof(uint16_t) * size_t(N) * K));
      SS_CUDA(cudaMalloc(&dc, sizeof(float) * size_t(M) * N));
      SS_CUDA(cudaMemcpyAsync(da, a, sizeof(uint16_t) * size_t(M) * K, cudaMemcpyHostToDevice, e->stream));
      SS_CUDA(cudaMemcpyAsync(db, b, sizeof(uint16_t) * size_t(N) * K, cudaMemcpyHostToDevice, e->stream));
      Gemm g = make_gemm(EPI_F32, da, db, M, N, K, e->dev_flags + 8, splitk_for(M, K));
      g.args.out_f32 = dc;
      if (g.args.splits > 1) {
        SS_CUDA(cudaMalloc(&dp, sizeof(float) * size_t(g.args.splits) * M * N));
        g.args.partial = dp;
      }
      launch_gemm(e, g);
      SS_CUDA(cudaMemcpyAsync(c, dc, sizeof(float) * size_t(M) * N, cudaMemcpyDeviceToHost, e->stream));
      sync(e);
      int flag = 0;
      SS_CUDA(cudaMemcpy(&flag, e->dev_flags + 8, sizeof(int), cudaMemcpyDeviceToHost));
      if (flag) {
        SS_CUDA(cudaMemset(e->dev_flags + 8, 0, sizeof(int)));
        fail(SS_ERR_TIMEOUT, "a tensor-core GEMM wait timed out");
      }
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

}  // extern "C"
