// Learned warm start: BF16 tensor-core GEMMs (tcgen05 + TMEM, TMA operand
// loads) with the epilogues the MLP's forward and backward passes need, plus
// the small kernels around them (feature gather/normalise with transpose,
// column sums, Adam, column statistics).
//
// GEMM shape: C[M x N] = A[M x K] * B[N x K]^T with A and B row-major and
// K-contiguous ("TN"), M tiled by 128 rows per CTA, N <= 256 per CTA, K in
// chunks of 64 (one 128-byte swizzle row per tile row).  Warp 0 lane 0 issues
// TMA loads into a 3-stage ring, warp 1 lane 0 issues tcgen05.mma (M 128,
// N = tile, K 16 per instruction) accumulating in TMEM, and all four warps
// read their 32 TMEM lanes back for the fused epilogue.  Every mbarrier wait
// is bounded by the global timer; a wait that gives up sets an abort flag
// for the CTA and the caller's error word, and the CTA skips the epilogue,
// releases its TMEM and returns.
#include "mlp_kernels.cuh"

#include <mutex>

namespace mjb {
namespace {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int STAGES = 3;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Waits for the phase with the given parity; false when the CTA aborted or
// the time limit passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, unsigned long long limit_ns = kWaitLimitNs) {
  const uint32_t addr = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; it++) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort_flag) return false;
    if ((it & 63) == 0) {
      unsigned long long t = global_ns();
      if (it == 0) t0 = t;
      else if (t - t0 > limit_ns) return false;
    }
  }
}

// Waits until the device word *flag is nonzero; false when the CTA aborted
// or the time limit passed.
__device__ __forceinline__ bool flag_wait(const volatile int* flag, volatile int* abort_flag, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (*flag != 0) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 128 bytes, 8-row groups 1024 bytes apart (SBO), LBO unused (1), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
        "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ void store_row16(__nv_bfloat16* dst, const float* v) {
  __align__(16) __nv_bfloat162 h[8];
#pragma unroll
  for (int i = 0; i < 8; i++) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  uint4* d = reinterpret_cast<uint4*>(dst);
  const uint4* s = reinterpret_cast<const uint4*>(h);
  d[0] = s[0];
  d[1] = s[1];
}

template <int BN>
__global__ void __launch_bounds__(128, 1) gemm_tn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs a) {
  constexpr int A_BYTES = BM * BK * 2;
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  // this CTA's K chunks: all of them, or slice blockIdx.z of ksplit
  const int nks = a.ksplit > 1 ? a.ksplit : 1;
  const int kc0 = (a.K / BK) * (int)blockIdx.z / nks;
  const int nk = (a.K / BK) * ((int)blockIdx.z + 1) / nks - kc0;
  float* const out_f32 = a.ksplit > 1 ? a.split_ws + (size_t)blockIdx.z * a.M * a.ldo : a.out_f32;
  const unsigned long long limit = a.wait_limit_ns ? a.wait_limit_ns : kWaitLimitNs;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  int issued = 0;
  if (warp == 0 && lane == 0) {
    for (int kc = 0; kc < nk; kc++) {
      const int s = kc % STAGES;
      if (kc >= STAGES && !mbar_wait(&empty[s], ((kc / STAGES) - 1) & 1, abort_flag, limit)) {
        *abort_flag = 1;
        break;
      }
      uint8_t* sa = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      tma_load_2d(sa, &tmA, &full[s], (kc0 + kc) * BK, m0);
      tma_load_2d(sa + A_BYTES, &tmB, &full[s], (kc0 + kc) * BK, n0);
      issued = kc + 1;
    }
  } else if (warp == 1 && lane == 0) {
    int nmma = 0;
    // test hook (a.gate): the first MMA waits for a device word; a word that
    // nothing sets makes this bounded wait run out and the CTA abort
    if (a.gate && !flag_wait(a.gate, abort_flag, limit)) *abort_flag = 1;
    for (int kc = 0; kc < nk && !*abort_flag; kc++) {
      const int s = kc % STAGES;
      if (!mbar_wait(&full[s], (kc / STAGES) & 1, abort_flag, limit)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t sb = sa + A_BYTES;
#pragma unroll
      for (int k = 0; k < BK / 16; k++) mma_bf16(tmem, sw128_desc(sa + 32 * k), sw128_desc(sb + 32 * k), IDESC, (kc | k) != 0);
      mma_commit(&empty[s]);
      nmma++;
    }
    // done completes once every MMA issued here has finished (a plain
    // arrive when none was issued)
    if (nmma) mma_commit(done);
    else mbar_arrive(done);
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0, abort_flag, limit) && !*abort_flag;
  __syncwarp();
  tc_fence_after();

  if (ok) {
    const int row = m0 + warp * 32 + lane;
    const bool rv = row < a.M;
    const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
    float lsum = 0.f;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + c0, v);
      const int col0 = n0 + c0;
      if (col0 >= a.N) continue;  // warp-uniform
      if (a.bias && a.mode != EPI_BWD_GELU) {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] += a.bias[col0 + i];
      }
      // rows past M store nothing; the warp stays converged for the next
      // tcgen05.ld (a .sync.aligned instruction)
      if (rv) switch (a.mode) {
        case EPI_F32: {
          float4* d = reinterpret_cast<float4*>(out_f32 + (size_t)row * a.ldo + col0);
#pragma unroll
          for (int i = 0; i < 4; i++) d[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
          break;
        }
        case EPI_HIDDEN: {
          if (a.pre) store_row16(a.pre + (size_t)row * a.ldo + col0, v);
#pragma unroll
          for (int i = 0; i < 16; i++) v[i] = gelu(v[i]);
          store_row16(a.out + (size_t)row * a.ldo + col0, v);
          if (a.out_t) {
#pragma unroll
            for (int i = 0; i < 16; i++) a.out_t[(size_t)(col0 + i) * a.ldt + row] = __float2bfloat16_rn(v[i]);
          }
          break;
        }
        case EPI_OUT_LOSS: {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int col = col0 + i;
            float d = 0.f;
            if (col < a.nvalid) {
              d = v[i] - a.target[(size_t)row * a.nvalid + col];
              lsum += d * d;
            }
            v[i] = a.scale * d;
          }
          store_row16(a.out + (size_t)row * a.ldo + col0, v);
          if (a.out_t) {
#pragma unroll
            for (int i = 0; i < 16; i++) a.out_t[(size_t)(col0 + i) * a.ldt + row] = __float2bfloat16_rn(v[i]);
          }
          break;
        }
        case EPI_OUT_PRED: {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int col = col0 + i;
            if (col < a.nvalid) {
              const size_t o = (size_t)row * a.nvalid + col;
              a.pred[o] = a.prev[o] + a.omean[col] + a.ostd[col] * v[i];
            }
          }
          break;
        }
        case EPI_BWD_GELU: {
          const __nv_bfloat16* z = a.pre_in + (size_t)row * a.ldo + col0;
#pragma unroll
          for (int i = 0; i < 16; i++) v[i] *= gelu_grad(__bfloat162float(z[i]));
          store_row16(a.out + (size_t)row * a.ldo + col0, v);
          if (a.out_t) {
#pragma unroll
            for (int i = 0; i < 16; i++) a.out_t[(size_t)(col0 + i) * a.ldt + row] = __float2bfloat16_rn(v[i]);
          }
          break;
        }
        default:
          break;
      }
      __syncwarp();
    }
    if (a.mode == EPI_OUT_LOSS && a.loss) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
      if (lane == 0) atomicAdd(a.loss, lsum);
    }
  } else if (threadIdx.x == 0) {
    if (a.err) atomicExch(a.err, 1);
    // let the TMA copies this thread issued land, and the MMAs already
    // issued finish, before the CTA's shared memory and TMEM are released
    // (each wait again bounded by the time limit)
    volatile int no_abort = 0;
    for (int kc = issued > STAGES ? issued - STAGES : 0; kc < issued; kc++) mbar_wait(&full[kc % STAGES], (kc / STAGES) & 1, &no_abort, limit);
    mbar_wait(done, 0, &no_abort, limit);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

template <int BN>
size_t gemm_smem_bytes() {
  return 1024 + (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) + 128;
}

template <int BN>
cudaError_t launch_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmArgs& a, cudaStream_t s) {
  const size_t smem = gemm_smem_bytes<BN>();
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [&] { attr_err = cudaFuncSetAttribute(gemm_tn_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); });
  if (attr_err != cudaSuccess) return attr_err;
  dim3 grid((a.M + BM - 1) / BM, (a.N + BN - 1) / BN, a.ksplit > 1 ? a.ksplit : 1);
  gemm_tn_kernel<BN><<<grid, 128, smem, s>>>(tmA, tmB, a);
  return cudaGetLastError();
}

// out[r * ldo + c] = sum over z < nsplit, in order, of ws[z * M * ldo + r * ldo + c]
// for r < M, c < N (N a multiple of 4; one thread per 4 columns)
__global__ void __launch_bounds__(256) splitk_reduce_kernel(const float* ws, int nsplit, int M, int N, int ldo, float* out) {
  const int nq = N >> 2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M * nq) return;
  const int r = t / nq, c = (t - r * nq) << 2;
  const size_t o = (size_t)r * ldo + c, slice = (size_t)M * ldo;
  float4 acc = *reinterpret_cast<const float4*>(ws + o);
#pragma unroll 1
  for (int z = 1; z < nsplit; z++) {
    const float4 v = *reinterpret_cast<const float4*>(ws + z * slice + o);
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
    acc.w += v.w;
  }
  *reinterpret_cast<float4*>(out + o) = acc;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

}  // namespace

bool make_tmap_bf16(CUtensorMap* map, const void* base, int rows, int cols, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || !base || rows <= 0 || cols <= 0 || cols % BK != 0 || box_rows <= 0 || box_rows > 256) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t gemm_tn(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmArgs& a, cudaStream_t s) {
  if (a.M <= 0 || a.K <= 0 || a.K % BK != 0 || a.N <= 0 || a.N % 16 != 0) return cudaErrorInvalidValue;
  if (a.ksplit > 1 && (a.mode != EPI_F32 || a.bias || !a.split_ws || !a.out_f32 || a.ksplit > a.K / BK || a.ldo % 4 != 0))
    return cudaErrorInvalidValue;
  if (a.bn && (a.bn != 64 && a.bn != 128 && a.bn != 256)) return cudaErrorInvalidValue;
  if (a.bn && a.N % a.bn != 0) return cudaErrorInvalidValue;
  cudaError_t e = cudaErrorInvalidValue;
  if (a.bn == 64) e = launch_gemm<64>(tmA, tmB, a, s);
  else if (a.bn == 128) e = launch_gemm<128>(tmA, tmB, a, s);
  else if (a.N == 64) e = launch_gemm<64>(tmA, tmB, a, s);
  else if (a.N == 128) e = launch_gemm<128>(tmA, tmB, a, s);
  else if (a.N == 192) e = launch_gemm<192>(tmA, tmB, a, s);
  else if (a.N % 256 == 0) e = launch_gemm<256>(tmA, tmB, a, s);
  if (e != cudaSuccess || a.ksplit <= 1) return e;
  const int threads = a.M * (a.N / 4);
  splitk_reduce_kernel<<<(threads + 255) / 256, 256, 0, s>>>(a.split_ws, a.ksplit, a.M, a.N, a.ldo, a.out_f32);
  return cudaGetLastError();
}

int gemm_ksplit(int M, int N, int K) {
  // enough CTAs to spread the K loop over the SMs, at least 4 K chunks
  // (of 64) each so the 3-stage load ring still fills
  const int tiles = ((M + BM - 1) / BM) * ((N + 255) / 256);
  const int nk = K / BK;
  int ks = 1;
  while (ks * 2 * tiles <= 148 && nk / (ks * 2) >= 4) ks *= 2;
  return ks;
}

}  // namespace mjb

// ---------------------------------------------------------------- helpers

namespace mjb {
namespace {

constexpr int GATHER_ROWS = 64;

// One CTA normalises GATHER_ROWS rows into bf16: row r of the output takes
// raw source row src_row (idx[r] or r) = [a (na floats) | b (nb floats)],
// x_j = (raw_j - mean_j) * istd_j, zero past na + nb up to ld.  Writes the
// row-major tile and, when xt is given, its transpose (xt[j * ldt + r]), both
// coalesced through a shared-memory tile.  With targets: t[r][k] =
// (traw[src][k] - tmean[k]) * tistd[k].
__global__ void __launch_bounds__(256) gather_kernel(int rows, const int* idx, const float* a, int lda, int na, const float* b, int ldb, int nb,
                                                     const float* mean, const float* istd, __nv_bfloat16* x, int ld, __nv_bfloat16* xt, int ldt,
                                                     const float* traw, int nt, const float* tmean, const float* tistd, float* t) {
  extern __shared__ __nv_bfloat16 tile[];  // [GATHER_ROWS][ld + 2]
  const int r0 = blockIdx.x * GATHER_ROWS;
  const int pitch = ld + 2;
  for (int e = threadIdx.x; e < GATHER_ROWS * ld; e += blockDim.x) {
    const int rr = e / ld, j = e % ld, r = r0 + rr;
    float v = 0.f;
    if (r < rows) {
      const size_t src = idx ? (size_t)idx[r] : (size_t)r;
      if (j < na) v = (a[src * lda + j] - mean[j]) * istd[j];
      else if (j < na + nb) v = (b[src * ldb + (j - na)] - mean[j]) * istd[j];
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    tile[rr * pitch + j] = h;
    if (r < rows) x[(size_t)r * ld + j] = h;
  }
  if (t) {
    for (int e = threadIdx.x; e < GATHER_ROWS * nt; e += blockDim.x) {
      const int rr = e / nt, k = e % nt, r = r0 + rr;
      if (r >= rows) continue;
      const size_t src = idx ? (size_t)idx[r] : (size_t)r;
      t[(size_t)r * nt + k] = (traw[src * nt + k] - tmean[k]) * tistd[k];
    }
  }
  if (!xt) return;
  __syncthreads();
  for (int e = threadIdx.x; e < GATHER_ROWS * ld; e += blockDim.x) {
    const int j = e / GATHER_ROWS, rr = e % GATHER_ROWS, r = r0 + rr;
    if (r < rows) xt[(size_t)j * ldt + r] = tile[rr * pitch + j];
  }
}

// out[j] = sum_r g[j * ld + r] over r < n (one CTA per j).
__global__ void __launch_bounds__(256) rowsum_kernel(const __nv_bfloat16* g, int ld, int n, float* out) {
  const int j = blockIdx.x;
  float s = 0.f;
  for (int r = threadIdx.x; r < n; r += blockDim.x) s += __bfloat162float(g[(size_t)j * ld + r]);
  __shared__ float red[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    out[j] = t;
  }
}

// Adam on n fp32 parameters; for a weight matrix [rows][cols] also writes the
// bf16 copy w and its transpose wt (either may be null).
__global__ void adam_kernel(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, float bc1, float bc2,
                            float wd, int rows, int cols, __nv_bfloat16* w, __nv_bfloat16* wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float pi = p[i] - lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * p[i]);
  p[i] = pi;
  if (w) w[i] = __float2bfloat16_rn(pi);
  if (wt) {
    const int r = i / cols, c = i % cols;
    wt[(size_t)c * rows + r] = __float2bfloat16_rn(pi);
  }
  (void)rows;
}

// Column sums and sums of squares of x[n][c] (double accumulators).
__global__ void __launch_bounds__(256) colstats_kernel(const float* x, int n, int c, int ld, double* sum, double* sq) {
  for (int j = threadIdx.x; j < c; j += blockDim.x) {
    double s = 0, q = 0;
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
      const double v = x[(size_t)r * ld + j];
      s += v;
      q += v * v;
    }
    atomicAdd(sum + j, s);
    atomicAdd(sq + j, q);
  }
}

// w[i] = bf16(p[i]) and the transpose, for uploading initial weights.
__global__ void cast_weights_kernel(int rows, int cols, const float* p, __nv_bfloat16* w, __nv_bfloat16* wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const __nv_bfloat16 h = __float2bfloat16_rn(p[i]);
  w[i] = h;
  if (wt) wt[(size_t)(i % cols) * rows + i / cols] = h;
}

}  // namespace

cudaError_t gather_rows(int rows, const int* idx, const float* a, int lda, int na, const float* b, int ldb, int nb, const float* mean, const float* istd,
                        __nv_bfloat16* x, int ld, __nv_bfloat16* xt, int ldt, const float* traw, int nt, const float* tmean, const float* tistd,
                        float* t, cudaStream_t s) {
  if (rows <= 0) return cudaSuccess;
  const size_t smem = (size_t)GATHER_ROWS * (ld + 2) * sizeof(__nv_bfloat16);
  static std::once_flag once;
  std::call_once(once, [] { cudaFuncSetAttribute(gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024); });
  if (smem > 64 * 1024) return cudaErrorInvalidValue;
  gather_kernel<<<(rows + GATHER_ROWS - 1) / GATHER_ROWS, 256, smem, s>>>(rows, idx, a, lda, na, b, ldb, nb, mean, istd, x, ld, xt, ldt, traw, nt,
                                                                            tmean, tistd, t);
  return cudaGetLastError();
}

cudaError_t rowsum_bf16(const __nv_bfloat16* g, int rows, int ld, int n, float* out, cudaStream_t s) {
  rowsum_kernel<<<rows, 256, 0, s>>>(g, ld, n, out);
  return cudaGetLastError();
}

cudaError_t adam_step(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, int t, float wd, int rows, int cols,
                      __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s) {
  const float bc1 = 1.f - powf(b1, (float)t), bc2 = 1.f - powf(b2, (float)t);
  adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, p, g, m, v, lr, b1, b2, eps, bc1, bc2, wd, rows, cols, w, wt);
  return cudaGetLastError();
}

cudaError_t column_stats(const float* x, int n, int c, int ld, double* sum, double* sq, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(sum, 0, sizeof(double) * c, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(sq, 0, sizeof(double) * c, s);
  if (e != cudaSuccess) return e;
  colstats_kernel<<<256, 256, 0, s>>>(x, n, c, ld, sum, sq);
  return cudaGetLastError();
}

cudaError_t cast_weights(int rows, int cols, const float* p, __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s) {
  cast_weights_kernel<<<(rows * cols + 255) / 256, 256, 0, s>>>(rows, cols, p, w, wt);
  return cudaGetLastError();
}

}  // namespace mjb

// ------------------------------------------------------- fused inference

namespace mjb {
namespace {

constexpr int INF_ACT_BYTES = 128 * 256 * 2;     // 128 rows x up to 256 bf16, 4 K-chunks of 16 KB
constexpr int INF_STAGE_BYTES = 256 * 64 * 2;    // one 64-wide K-chunk of up to 256 weight rows
constexpr int INF_STAGES = 2;

// Byte offset of element (row r, column j) in the chunked, 128-byte
// swizzled K-major operand layout (chunk = 64 columns x 128 rows).
__device__ __forceinline__ uint32_t act_off(int r, int j) {
  const int c = j >> 6, jj = j & 63;
  return (uint32_t)(c * 16384 + r * 128 + ((((jj >> 3) ^ (r & 7)) & 7) << 4) + (jj & 7) * 2);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
}

// One CTA computes the warm-start prediction of 128 envs: gather and
// normalise [features | controls] into bf16 (shared memory, UMMA operand
// layout), then for each layer: stream the weight K-chunks through a 2-stage
// TMA ring, tcgen05.mma into TMEM, and write bias + GELU activations back
// over the operand buffer; the output layer writes prev + mean + std * y.
__global__ void __launch_bounds__(128, 1) mlp_infer_kernel(const __grid_constant__ CUtensorMap w0, const __grid_constant__ CUtensorMap w1,
                                                           const __grid_constant__ CUtensorMap w2, const __grid_constant__ CUtensorMap w3,
                                                           InferArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* act = smem;
  uint8_t* ring = smem + INF_ACT_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + INF_STAGES * INF_STAGE_BYTES);
  uint64_t* empty = full + INF_STAGES;
  uint64_t* done = empty + INF_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const CUtensorMap* maps[4] = {&w0, &w1, &w2, &w3};

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128;
  const uint32_t act_s = smem_u32(act);

  if (threadIdx.x == 0) {
    for (int s = 0; s < INF_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(256u) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // gather + normalise: warp w fills rows 32w .. 32w+31; lane handles the
  // columns lane + 32k; 4 rows per pass keep up to 32 independent loads per
  // lane in flight (the gather is latency bound otherwise)
  {
    const int kmax = a.in_pad >> 5, nin = a.nfeat + a.nu;
    float mu[8], is[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int j = lane + 32 * k;
      mu[k] = (k < kmax && j < nin) ? a.mean[j] : 0.f;
      is[k] = (k < kmax && j < nin) ? a.istd[j] : 0.f;
    }
#pragma unroll 1
    for (int rr = 0; rr < 32; rr += 4) {
      float v[4][8];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int env = m0 + warp * 32 + rr + q;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int j = lane + 32 * k;
          float x = 0.f;
          if (k < kmax && env < a.B) {
            if (j < a.nfeat) x = __ldg(a.feat + (size_t)env * a.fstride + j);
            else if (j < nin) x = __ldg(a.ctrl + (size_t)env * a.nu + (j - a.nfeat));
          }
          v[q][k] = x;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = warp * 32 + rr + q;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          if (k < kmax) {
            const int j = lane + 32 * k;
            *reinterpret_cast<__nv_bfloat16*>(act + act_off(r, j)) = __float2bfloat16_rn((v[q][k] - mu[k]) * is[k]);
          }
        }
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  int g = 0;  // K-chunk counter over all layers (ring stage and phase)
  int issued = 0;   // chunks whose TMA load thread 0 issued (thread 0 only)
  int lfail = 0;    // layer whose wait gave up
  bool ok = true;
#pragma unroll 1
  for (int l = 0; l < 4 && ok; l++) {
    const int N = a.rows[l], K = a.cols[l], nk = K / 64;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    if (warp == 0 && lane == 0) {
      for (int c = 0; c < nk; c++) {
        const int gc = g + c, s = gc % INF_STAGES;
        if (gc >= INF_STAGES && !mbar_wait(&empty[s], ((gc / INF_STAGES) - 1) & 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        mbar_expect_tx(&full[s], (uint32_t)(N * 128));
        tma_load_2d(ring + s * INF_STAGE_BYTES, maps[l], &full[s], c * 64, 0);
        issued = gc + 1;
      }
    } else if (warp == 1 && lane == 0) {
      int nmma = 0;
      for (int c = 0; c < nk; c++) {
        const int gc = g + c, s = gc % INF_STAGES;
        if (!mbar_wait(&full[s], (gc / INF_STAGES) & 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t sa = act_s + c * 16384;
        const uint32_t sb = smem_u32(ring + s * INF_STAGE_BYTES);
#pragma unroll
        for (int k = 0; k < 4; k++) mma_bf16(tmem, sw128_desc(sa + 32 * k), sw128_desc(sb + 32 * k), idesc, (c | k) != 0);
        mma_commit(&empty[s]);
        nmma++;
      }
      // this layer's phase of done completes once its MMAs have finished
      // (a plain arrive when none was issued)
      if (nmma) mma_commit(done);
      else mbar_arrive(done);
    }
    g += nk;
    __syncwarp();
    ok = mbar_wait(done, l & 1, abort_flag) && !*abort_flag;
    __syncwarp();
    tc_fence_after();
    if (!ok) {
      lfail = l;
      break;
    }
    // epilogue: TMEM lanes of this warp = its 32 rows
    const int r = warp * 32 + lane, env = m0 + r;
    const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
    const float* bias = a.bias[l];
#pragma unroll 1
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + c0, v);
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] += bias[c0 + i];
      if (l < 3) {
        __align__(16) __nv_bfloat162 h[8];
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = __floats2bfloat162_rn(gelu(v[2 * i]), gelu(v[2 * i + 1]));
        const uint4* hv = reinterpret_cast<const uint4*>(h);
        st_shared_v4(act_s + act_off(r, c0), hv[0]);
        st_shared_v4(act_s + act_off(r, c0 + 8), hv[1]);
      } else if (env < a.B) {
#pragma unroll
        for (int i = 0; i < 16; i++) {
          const int k = c0 + i;
          if (k < a.nout) {
            const size_t o = (size_t)env * a.nout + k;
            a.pred[o] = a.prev[o] + a.omean[k] + a.ostd[k] * v[i];
          }
        }
      }
      __syncwarp();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok && threadIdx.x == 0) {
    if (a.err) atomicExch(a.err, 2);
    // let the TMA copies this thread issued land, and the layer's MMAs
    // finish, before the CTA's shared memory and TMEM are released (each
    // wait bounded by the time limit)
    volatile int no_abort = 0;
    for (int gc = issued > INF_STAGES ? issued - INF_STAGES : 0; gc < issued; gc++)
      mbar_wait(&full[gc % INF_STAGES], (gc / INF_STAGES) & 1, &no_abort);
    mbar_wait(done, lfail & 1, &no_abort);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
  }
}

}  // namespace

cudaError_t mlp_infer(const CUtensorMap* wmaps, const InferArgs& a, cudaStream_t s) {
  if (a.B <= 0) return cudaSuccess;
  if (a.in_pad > 256 || a.in_pad % 64 != 0) return cudaErrorInvalidValue;
  for (int l = 0; l < 4; l++)
    if (a.rows[l] > 256 || a.rows[l] % 16 != 0 || a.cols[l] % 64 != 0 || a.cols[l] > 256) return cudaErrorInvalidValue;
  const size_t smem = 1024 + INF_ACT_BYTES + INF_STAGES * INF_STAGE_BYTES + 128;
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [&] { attr_err = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); });
  if (attr_err != cudaSuccess) return attr_err;
  mlp_infer_kernel<<<(a.B + 127) / 128, 128, smem, s>>>(wmaps[0], wmaps[1], wmaps[2], wmaps[3], a);
  return cudaGetLastError();
}

}  // namespace mjb
