// Shared declarations of the learned warm-start kernels (BF16 tcgen05 GEMMs
// with fused epilogues, feature gathers, reductions, Adam).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mjb {

// Epilogue of C[M x N] = A[M x K] * B[N x K]^T (both operands K-contiguous).
enum GemmEpilogue : int {
  EPI_F32 = 0,          // out_f32[row * ldo + col] = acc (+ bias when given)
  EPI_HIDDEN = 1,       // z = acc + bias; pre = bf16(z) (optional); out = bf16(gelu(z)); out_t = transposed out (optional)
  EPI_OUT_LOSS = 2,     // y = acc + bias; d = y - target (cols < nvalid); loss += sum d^2; out / out_t = bf16(scale * d)
  EPI_OUT_PRED = 3,     // y = acc + bias; pred[row * nvalid + col] = prev[...] + omean[col] + ostd[col] * y   (cols < nvalid)
  EPI_BWD_GELU = 4,     // dz = acc * gelu'(pre_in); out = bf16(dz); out_t = transposed (optional)
};

struct GemmArgs {
  int M, N, K;          // N: columns computed (multiple of 16, <= 256 per CTA tile); K multiple of 64
  int mode;
  int ldo;              // leading dimension of out / out_f32 / pre / pre_in (elements)
  int ldt;              // leading dimension of out_t (>= M)
  int nvalid;           // EPI_OUT_*: number of real output columns
  const float* bias;    // [N] or null
  float* out_f32;
  __nv_bfloat16* out;
  __nv_bfloat16* out_t;
  __nv_bfloat16* pre;
  const __nv_bfloat16* pre_in;
  const float* target;  // EPI_OUT_LOSS: [M][nvalid]
  float* loss;          // EPI_OUT_LOSS: accumulated sum of squares
  float scale;          // EPI_OUT_LOSS: gradient scale
  const float* prev;    // EPI_OUT_PRED: [M][nvalid]
  const float* omean;
  const float* ostd;
  float* pred;
  int* err;             // set to a nonzero code when a bounded wait gives up
  const volatile int* gate;       // test hook (null in production): the first MMA waits, bounded, for *gate != 0
  unsigned long long wait_limit_ns;  // limit of each bounded wait (0: 2 s)
  // split K (EPI_F32 without bias only): ksplit > 1 CTAs share each output
  // tile, each over a contiguous range of the K chunks, writing FP32 partial
  // tiles into split_ws (ksplit slices of M x ldo floats); a second kernel
  // sums the slices in slice order into out_f32, so results do not depend
  // on scheduling.  Used for the weight gradients, whose K is the batch.
  int ksplit;
  float* split_ws;
  // N tile width of the launch: 0 picks the widest N allows (one CTA per 256
  // columns); 64 or 128 give more, narrower CTAs (for small M).  tmB's box
  // must have this many rows.
  int bn;
};

// Encodes a 2-D bf16 row-major [rows][cols] tensor map with a box of
// {64, box_rows} and 128-byte swizzle (zero fill outside the tensor).
bool make_tmap_bf16(CUtensorMap* map, const void* base, int rows, int cols, int box_rows);

// Launches the tcgen05 GEMM for C[M x N] = A * B^T.  tmA: A [M][K] with box
// rows 128; tmB: B [N][K] with box rows = the CTA's N tile (N <= 256 in one
// tile, else 256-column tiles).
cudaError_t gemm_tn(const CUtensorMap& tmA, const CUtensorMap& tmB, const GemmArgs& a, cudaStream_t s);
// Split of the K loop gemm_tn should use for an EPI_F32 C[M x N] with this
// K (a power of two, 1 when the tiles alone fill the GPU).
int gemm_ksplit(int M, int N, int K);

}  // namespace mjb

namespace mjb {

// Normalising gather into bf16 rows (and optionally their transpose) plus
// normalised targets; see gather_kernel.
cudaError_t gather_rows(int rows, const int* idx, const float* a, int lda, int na, const float* b, int ldb, int nb, const float* mean, const float* istd,
                        __nv_bfloat16* x, int ld, __nv_bfloat16* xt, int ldt, const float* traw, int nt, const float* tmean, const float* tistd,
                        float* t, cudaStream_t s);
// out[j] = sum over r < n of g[j * ld + r], j < rows.
cudaError_t rowsum_bf16(const __nv_bfloat16* g, int rows, int ld, int n, float* out, cudaStream_t s);
// One Adam step (bias-corrected, decoupled weight decay wd) on n parameters;
// writes bf16 copies w ([rows][cols]) and wt (transpose) when given.
cudaError_t adam_step(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, int t, float wd, int rows, int cols,
                      __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s);
// Column sums / sums of squares of x[n][c] with row stride ld.
cudaError_t column_stats(const float* x, int n, int c, int ld, double* sum, double* sq, cudaStream_t s);
// bf16 copy of a fp32 weight matrix and its transpose.
cudaError_t cast_weights(int rows, int cols, const float* p, __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s);

// Fused warm-start inference (gather + normalise + 4 layers + prediction).
struct InferArgs {
  int B;                  // envs (rows)
  const float* feat;      // [B][fstride], first nfeat used
  int fstride, nfeat;
  const float* ctrl;      // [B][nu]
  int nu;
  int in_pad;             // padded input width (multiple of 64, <= 256)
  const float* mean;      // [nfeat + nu]
  const float* istd;
  int rows[4], cols[4];   // layer shapes (weights [rows][cols]); cols[0] = in_pad
  const float* bias[4];
  int nout;
  const float* prev;      // [B][nout]
  const float* omean;
  const float* ostd;
  float* pred;            // [B][nout]
  int* err;
};
// wmaps: tensor maps of the 4 bf16 weight matrices, box {64, rows[l]}.
cudaError_t mlp_infer(const CUtensorMap* wmaps, const InferArgs& a, cudaStream_t s);

}  // namespace mjb
