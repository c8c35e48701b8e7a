// Constraint rows, Newton solve and Euler integration for one env per warp.
//   d_constraints <- solver.hpp:259-587 (rows: frictionloss -> limits ->
//                    contacts; impedance efc_kbi :122-138; pyramid rows with
//                    R = 2 mu0^2/impratio * R_first :536-571)
//   d_newton      <- solver.hpp:592-854 (H = M + J'DJ, shared-memory Cholesky
//                    :743-785), with previous-step / predicted warm start,
//                    exact line search and tolerance-scaled termination
//   d_integrate   <- euler.hpp:26-110, batched.cpp:712-745 (implicit damping)
// Rows are added in order; the first row group that does not fit in
// nefc_max is dropped together with every later group (status bit set).
#pragma once
#include "dev_stages.cuh"

namespace mjbdev {

// Cholesky of the n x n SPD matrix A (row-major, lower triangle used, in
// place: L below the diagonal, L_jj on it); idiag[j] = 1 / L_jj.
// Right-looking: after column k is scaled, the m(m+1)/2 entries of the
// trailing lower triangle (m = n - k - 1) are spread evenly over the lanes,
// so every lane does about m^2 / 64 independent updates per step instead of
// the lane owning the last row doing m of them in sequence.
__device__ __noinline__ void d_chol_smem(float* A, int n, int lane, float* idiag) {
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    float d = sqrtf(fmaxf(A[k * n + k], 1e-30f));
    float id = 1.f / d;
    __syncwarp();
#pragma unroll 1
    for (int i = k + 1 + lane; i < n; i += 32) A[i * n + k] *= id;
    if (lane == 0) {
      A[k * n + k] = d;
      idiag[k] = id;
    }
    __syncwarp();
    const int m = n - k - 1, T = m * (m + 1) / 2, k1 = k + 1;
#pragma unroll 2
    for (int t = lane; t < T; t += 32) {
      // entry t of the trailing lower triangle in row-major order: row r with
      // r (r + 1) / 2 <= t < (r + 1) (r + 2) / 2, column t - r (r + 1) / 2
      int r = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
      if ((r + 1) * (r + 2) / 2 <= t) r++;
      else if (r * (r + 1) / 2 > t) r--;
      const int c = t - r * (r + 1) / 2;
      const int i = k1 + r, j = k1 + c;
      A[i * n + j] -= A[i * n + k] * A[j * n + k];
    }
    __syncwarp();
  }
}

// Cholesky for n <= 32 with rows padded to ld floats (a multiple of 4) and
// col[32] (16-byte aligned) of scratch.  At step k lane i > k scales its
// entry k and posts it to col[i]; every lane then updates its own row's
// entries k+1..i four at a time with 16-byte loads and stores, reading the
// posted column with broadcast loads instead of one shuffle per entry.  The
// last group of a row may reach past its diagonal into the padded upper
// triangle, which nothing reads.  The updates are d_chol_smem's in the same
// order; the pivot's 1 / sqrt is the hardware estimate refined by one Newton
// step instead of IEEE sqrt and division.
__device__ __noinline__ void d_chol_vec(float* A, int n, int ld, int lane, float* idiag, float* col) {
  const bool own = lane < n;
  float* row = A + lane * ld;
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    // pivot: 1 / sqrt from the hardware estimate plus one Newton step
    // (about 1 ulp), d = akk / sqrt(akk)
    const float akk = fmaxf(A[k * ld + k], 1e-30f);
    float id = rsqrtf(akk);
    id = id * fmaf(-0.5f * akk * id, id, 1.5f);
    const float d = akk * id;
    const bool below = own && lane > k;
    float l = 0.f;
    if (below) {
      l = row[k] * id;
      row[k] = l;
      col[lane] = l;
    }
    if (lane == k) {
      row[k] = d;
      idiag[k] = id;
    }
    __syncwarp();
    if (below) {
#pragma unroll 1
      for (int j = (k + 1) & ~3; j <= lane; j += 4) {
        float4 a = *reinterpret_cast<float4*>(row + j);
        const float4 c = *reinterpret_cast<const float4*>(col + j);
        if (j > k) a.x -= l * c.x;
        if (j + 1 > k) a.y -= l * c.y;
        if (j + 2 > k) a.z -= l * c.z;
        a.w -= l * c.w;   // j + 3 > k always (j >= k - 2)
        *reinterpret_cast<float4*>(row + j) = a;
      }
    }
    __syncwarp();
  }
}

// Right-looking Cholesky that skips exact zeros (large models): after
// column k is scaled, its nonzero rows below the diagonal are listed with a
// ballot scan and only their pairs are updated.  The arithmetic on the
// nonzero entries is the dense algorithm's; for the bin of free bodies M is
// 6 x 6 block-diagonal and H keeps the contact graph's block pattern plus
// fill-in, so most of the n^3 / 6 updates of the dense version vanish.
// nz: n ints of scratch.
__device__ __noinline__ void d_chol_sparse(float* A, int n, int lane, float* idiag, int* nz) {
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    const float d = sqrtf(fmaxf(A[k * n + k], 1e-30f));
    const float id = 1.f / d;
    __syncwarp();
    int cnt = 0;
#pragma unroll 1
    for (int base = k + 1; base < n; base += 32) {
      const int i = base + lane;
      bool on = false;
      if (i < n) {
        const float v = A[i * n + k];
        on = v != 0.f;
        if (on) A[i * n + k] = v * id;
      }
      const unsigned bal = __ballot_sync(FULL_MASK, on);
      if (on) nz[cnt + __popc(bal & ((1u << lane) - 1u))] = i;
      cnt += __popc(bal);
    }
    if (lane == 0) {
      A[k * n + k] = d;
      idiag[k] = id;
    }
    __syncwarp();
    const int T = cnt * (cnt + 1) / 2;
#pragma unroll 1
    for (int t = lane; t < T; t += 32) {
      int p = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
      if ((p + 1) * (p + 2) / 2 <= t) p++;
      else if (p * (p + 1) / 2 > t) p--;
      const int q = t - p * (p + 1) / 2;
      const int i = nz[p], j = nz[q];
      A[i * n + j] -= A[i * n + k] * A[j * n + k];
    }
    __syncwarp();
  }
}

// ld: row stride of A (n rounded up to 4 for n <= 32, then col = A + n * ld
// is the vector path's column scratch; n otherwise)
__device__ __forceinline__ void d_chol(float* A, int n, int ld, int lane, float* idiag, int* nz = nullptr) {
  if (n <= 32) d_chol_vec(A, n, ld, lane, idiag, A + n * ld);
  else if (n > 64 && nz) d_chol_sparse(A, n, lane, idiag, nz);
  else d_chol_smem(A, n, lane, idiag);
}

// x := (L L')^-1 x.  The running vector lives in registers (element i on lane
// i; a second slot covers n up to 64) and each solved entry is broadcast with a
// shuffle, so the substitution needs no shared-memory round trip per step.
__device__ __noinline__ void d_chol_solve_mem(const float* L, const float* idiag, int n, float* x, int lane) {
  // n > 64: the running vector stays in the workspace, column by column
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    const float xk = x[k] * idiag[k];
    __syncwarp();
    if (lane == 0) x[k] = xk;
#pragma unroll 1
    for (int i = k + 1 + lane; i < n; i += 32) x[i] -= L[i * n + k] * xk;
    __syncwarp();
  }
#pragma unroll 1
  for (int k = n - 1; k >= 0; k--) {
    const float xk = x[k] * idiag[k];
    __syncwarp();
    if (lane == 0) x[k] = xk;
#pragma unroll 1
    for (int i = lane; i < k; i += 32) x[i] -= L[k * n + i] * xk;
    __syncwarp();
  }
}

// n <= 32 with rows padded to ld (a multiple of 4): the substitutions go
// four columns per group, loading the group's factor entries (one 16-byte
// row load forward, four row loads backward) and pivots before its four
// dependent shuffle steps, so the chain waits on shuffles only.  Same
// arithmetic in the same order as the general version.
__device__ __noinline__ void d_chol_solve32(const float* L, const float* idiag, int n, int ld, float* x, int lane) {
  const bool own = lane < n;
  float x0 = own ? x[lane] : 0.f;
  const float* Lr = L + lane * ld;
#pragma unroll 1
  for (int k0 = 0; k0 < n; k0 += 4) {
    const float4 lr = own ? *reinterpret_cast<const float4*>(Lr + k0) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float lq[4] = {lr.x, lr.y, lr.z, lr.w};
    float dg[4];
#pragma unroll
    for (int q = 0; q < 4; q++) dg[q] = k0 + q < n ? idiag[k0 + q] : 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int k = k0 + q;
      if (k >= n) break;
      const float xk = __shfl_sync(FULL_MASK, x0, k) * dg[q];
      if (lane == k) x0 = xk;
      else if (lane > k) x0 -= lq[q] * xk;
    }
  }
#pragma unroll 1
  for (int k0 = n - 1; k0 >= 0; k0 -= 4) {
    float lk[4], dg[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int k = k0 - q;
      lk[q] = k >= 0 && lane < k ? L[k * ld + lane] : 0.f;
      dg[q] = k >= 0 ? idiag[k] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int k = k0 - q;
      if (k < 0) break;
      const float xk = __shfl_sync(FULL_MASK, x0, k) * dg[q];
      if (lane == k) x0 = xk;
      else if (lane < k) x0 -= lk[q] * xk;
    }
  }
  if (own) x[lane] = x0;
  __syncwarp();
}

__device__ __noinline__ void d_chol_solve(const float* L, const float* idiag, int n, int ld, float* x, int lane) {
  if (n > 64) {
    d_chol_solve_mem(L, idiag, n, x, lane);
    return;
  }
  if (n <= 32) {
    d_chol_solve32(L, idiag, n, ld, x, lane);
    return;
  }
  float x0 = lane < n ? x[lane] : 0.f;
  float x1 = lane + 32 < n ? x[lane + 32] : 0.f;
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    float v = k < 32 ? __shfl_sync(FULL_MASK, x0, k) : __shfl_sync(FULL_MASK, x1, k - 32);
    float xk = v * idiag[k];
    if (lane == (k & 31)) {
      if (k < 32) x0 = xk;
      else x1 = xk;
    }
    if (lane > k && lane < n) x0 -= L[lane * ld + k] * xk;
    if (lane + 32 > k && lane + 32 < n) x1 -= L[(lane + 32) * ld + k] * xk;
  }
#pragma unroll 1
  for (int k = n - 1; k >= 0; k--) {
    float v = k < 32 ? __shfl_sync(FULL_MASK, x0, k) : __shfl_sync(FULL_MASK, x1, k - 32);
    float xk = v * idiag[k];
    if (lane == (k & 31)) {
      if (k < 32) x0 = xk;
      else x1 = xk;
    }
    if (lane < k && lane < n) x0 -= L[k * ld + lane] * xk;
    if (lane + 32 < k && lane + 32 < n) x1 -= L[k * ld + lane + 32] * xk;
  }
  if (lane < n) x[lane] = x0;
  if (lane + 32 < n) x[lane + 32] = x1;
  __syncwarp();
}

// Explicit inverses N = A^-1 for n <= 32 (full storage, rows padded to
// ld, a multiple of 4, with zeros past column n; row i on lane i).

// In-place inversion by the symmetric sweep operator on every pivot.  Step
// k: d = a_kk; every row i != k becomes a_i - (a_ik / d) a_k with entry k set
// to -a_ik / d; row k becomes a_k / d with entry k = 1 / d.  After all n
// steps A holds A^-1 whatever the pivot order.  The pivots are Schur
// complements of an SPD matrix, so they stay positive and no pivoting is
// needed.  Pivots go from the last dof to the first: in the depth-first
// dof order of a kinematic tree that sweeps leaves before their ancestors,
// and a row with a_ik = 0 (a dof on another branch) is left as it is, so M
// and Hessians with the tree's pattern keep the branches apart until their
// common ancestors' pivots (for the quadruped a leg pivot touches the 9 rows
// of the free joint and its own leg instead of 18).  The pivot row is first
// copied to col (16-byte aligned, ld floats), so every lane, its owner
// included (factor 1 - 1/d gives a_k / d), updates its own row from the
// copy with 16-byte loads and stores.
__device__ __noinline__ void d_sweep(float* A, int n, int ld, int lane, float* col) {
  const bool own = lane < n;
  float* row = A + lane * ld;
#pragma unroll 1
  for (int k = n - 1; k >= 0; k--) {
    __syncwarp();
    if (lane < ld) col[lane] = A[k * ld + lane];
    __syncwarp();
    const float id = __frcp_rn(col[k]);
    const float aik = own ? row[k] : 0.f;
    if (own && (aik != 0.f || lane == k)) {
      const float f = lane == k ? 1.f - id : aik * id;
#pragma unroll 2
      for (int j = 0; j < ld; j += 4) {
        float4 a = *reinterpret_cast<float4*>(row + j);
        const float4 c = *reinterpret_cast<const float4*>(col + j);
        a.x = fmaf(-f, c.x, a.x);
        a.y = fmaf(-f, c.y, a.y);
        a.z = fmaf(-f, c.z, a.z);
        a.w = fmaf(-f, c.w, a.w);
        *reinterpret_cast<float4*>(row + j) = a;
      }
      row[k] = lane == k ? id : -f;
    }
  }
  __syncwarp();
}

// sum_j a[j] x[j] over ld floats (both 16-byte aligned)
__device__ __forceinline__ float row_dot4(const float* a, const float* x, int ld) {
  float s0 = 0.f, s1 = 0.f;
#pragma unroll 2
  for (int j = 0; j < ld; j += 4) {
    const float4 p = *reinterpret_cast<const float4*>(a + j);
    const float4 q = *reinterpret_cast<const float4*>(x + j);
    s0 = fmaf(p.x, q.x, s0);
    s1 = fmaf(p.y, q.y, s1);
    s0 = fmaf(p.z, q.z, s0);
    s1 = fmaf(p.w, q.w, s1);
  }
  return s0 + s1;
}

// y = N v for the inverse N (lane i returns y_i; lanes >= n return 0).
// col: 16-byte aligned scratch of ld floats, v: n floats.
__device__ __noinline__ float d_inv_apply(const float* N, int n, int ld, float* col, const float* v, int lane) {
  __syncwarp();
  if (lane < ld) col[lane] = lane < n ? v[lane] : 0.f;
  __syncwarp();
  const float y = lane < n ? row_dot4(N + lane * ld, col, ld) : 0.f;
  __syncwarp();
  return y;
}

// N = A^-1 updated for A + sgn x x' with x = w J_r (one constraint row),
// by Sherman-Morrison: u = N x, s = x'u, N -= sgn u u' / (1 + sgn s).  For
// an update the denominator is 1 + x'A^-1 x >= 1; for a downdate it is
// 1 - x'A^-1 x in (0, 1], and below 0.02 (the row carries nearly all of A
// along x, so the subtraction cancels and rounding errors grow by up to the
// reciprocal) the call returns false with N unchanged and the caller
// rebuilds the inverse.  Measured on the quadruped, bounds of 0.1 and 0.3
// rebuild more often and cost more time than the extra Newton iterations
// that the looser bound brings.
__device__ __noinline__ bool d_inv_rank1(float* N, int n, int ld, float* col, const float* Jr, float w, float sgn, int lane) {
  const bool own = lane < n;
  float* row = N + lane * ld;
  __syncwarp();
  const float x = own ? w * Jr[lane] : 0.f;
  if (lane < ld) col[lane] = x;
  __syncwarp();
  const float u = own ? row_dot4(row, col, ld) : 0.f;
  const float den = 1.f + sgn * warp_sum(x * u);
  if (!(den > 0.02f)) return false;
  const float gu = -sgn * __frcp_rn(den) * u;
  __syncwarp();
  if (lane < ld) col[lane] = u;
  __syncwarp();
  if (own) {
#pragma unroll 2
    for (int j = 0; j < ld; j += 4) {
      float4 a = *reinterpret_cast<float4*>(row + j);
      const float4 c = *reinterpret_cast<const float4*>(col + j);
      a.x = fmaf(gu, c.x, a.x);
      a.y = fmaf(gu, c.y, a.y);
      a.z = fmaf(gu, c.z, a.z);
      a.w = fmaf(gu, c.w, a.w);
      *reinterpret_cast<float4*>(row + j) = a;
    }
  }
  __syncwarp();
  return true;
}

// A = M + sum over the listed rows r of D_r J_r' J_r + dscale * diag(ddiag),
// built in shared memory entry by entry of the lower triangle (entries spread
// over the lanes, row and column computed from the entry index), then
// factored by the right-looking shared-memory Cholesky
// into the row-major lower triangle of L with idiag = 1 / L_jj.
// Middle-zone elliptic cones add A A' - W W' per cone (A = sum_a HA_a J_a,
// W = sum_a HU_a J_a over the cone's rows); their tangent rows' own terms
// come in through the active list with weight HD.  cones[-k] (k < ncone)
// holds normal row | dim << 16; hau = the HA field (HU follows at + ne).
__device__ __forceinline__ float cone_entry(const float* J, const float* hau, int ne, const int* cones, int ncone, int n, int i, int j) {
  float s = 0.f;
#pragma unroll 1
  for (int k = 0; k < ncone; k++) {
    const int code = cones[-k], r = code & 0xffff, dim = code >> 16;
    float Ai = 0.f, Aj = 0.f, Ui = 0.f, Uj = 0.f;
#pragma unroll 1
    for (int a = 0; a < dim; a++) {
      const float* Jr = J + (r + a) * n;
      const float ha = hau[r + a], hu = hau[ne + r + a], ji = Jr[i], jj = Jr[j];
      Ai += ha * ji;
      Aj += ha * jj;
      Ui += hu * ji;
      Uj += hu * jj;
    }
    s += Ai * Aj - Ui * Uj;
  }
  return s;
}

// inv = true (n <= 32, no cones): both triangles and zero padding are
// written and L receives N = A^-1 from the sweep instead of the factor.
__device__ __noinline__ void d_factor_smem(const float* M, const float* J, const float* eD, const int* act, int nact, const float* ddiag, float dscale,
                                           int n, int ld, int lane, float* L, float* idiag,
                                           const int* cones = nullptr, int ncone = 0, const float* hau = nullptr, int ne = 0, bool inv = false) {
  const int ntri = n * (n + 1) / 2;
#pragma unroll 1
  for (int t = lane; t < ntri; t += 32) {
    // entry t of the lower triangle in row-major order (row i, column j)
    int i = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
    if ((i + 1) * (i + 2) / 2 <= t) i++;
    else if (i * (i + 1) / 2 > t) i--;
    const int j = t - i * (i + 1) / 2;
    float s0 = M[i * n + j], s1 = 0, s2 = 0, s3 = 0;
    if (i == j && ddiag) s0 += dscale * ldf(ddiag, i);
    int a = 0;
#pragma unroll 1
    for (; a + 3 < nact; a += 4) {
      int r0 = act[a], r1 = act[a + 1], r2 = act[a + 2], r3 = act[a + 3];
      s0 += eD[r0] * J[r0 * n + i] * J[r0 * n + j];
      s1 += eD[r1] * J[r1 * n + i] * J[r1 * n + j];
      s2 += eD[r2] * J[r2 * n + i] * J[r2 * n + j];
      s3 += eD[r3] * J[r3 * n + i] * J[r3 * n + j];
    }
#pragma unroll 1
    for (; a < nact; a++) {
      int r0 = act[a];
      s0 += eD[r0] * J[r0 * n + i] * J[r0 * n + j];
    }
    if (ncone) s1 += cone_entry(J, hau, ne, cones, ncone, n, i, j);
    L[i * ld + j] = (s0 + s1) + (s2 + s3);
    if (inv) L[j * ld + i] = (s0 + s1) + (s2 + s3);
  }
  if (inv) {
#pragma unroll 1
    for (int i = lane; i < n; i += 32)
      for (int j = n; j < ld; j++) L[i * ld + j] = 0.f;
    __syncwarp();
    d_sweep(L, n, ld, lane, L + n * ld);
    return;
  }
  __syncwarp();
  d_chol(L, n, ld, lane, idiag);
}

// Row-sparse variant for large models (nv > 64, HBM workspaces): a contact
// row touches only the dofs of its two bodies' chains (12 for two free
// bodies out of hundreds), so H = M + sum D_r J_r' J_r is accumulated row by
// row over each row's nonzero columns (found with a ballot scan) instead of
// entry by entry over every active row.
__device__ __noinline__ void d_factor_sparse(const float* M, const float* J, const float* eD, const int* act, int nact, const float* ddiag, float dscale,
                                             int n, int lane, int* nz, float* L, float* idiag,
                                             const int* cones = nullptr, int ncone = 0, const float* hau = nullptr, int ne = 0) {
#pragma unroll 1
  for (int i = 0; i < n; i++) {
#pragma unroll 1
    for (int j = lane; j <= i; j += 32) L[i * n + j] = M[i * n + j] + ((i == j && ddiag) ? dscale * ldf(ddiag, i) : 0.f);
  }
  __syncwarp();
#pragma unroll 1
  for (int a = 0; a < nact; a++) {
    const int r = act[a];
    const float* row = J + r * n;
    int cnt = 0;
#pragma unroll 1
    for (int base = 0; base < n; base += 32) {
      const int c = base + lane;
      const bool on = c < n && row[c] != 0.f;
      const unsigned bal = __ballot_sync(FULL_MASK, on);
      if (on) nz[cnt + __popc(bal & ((1u << lane) - 1u))] = c;
      cnt += __popc(bal);
    }
    __syncwarp();
    const float d = eD[r];
    const int T = cnt * (cnt + 1) / 2;
#pragma unroll 1
    for (int t = lane; t < T; t += 32) {
      int p = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
      if ((p + 1) * (p + 2) / 2 <= t) p++;
      else if (p * (p + 1) / 2 > t) p--;
      const int q = t - p * (p + 1) / 2;
      const int i = nz[p], j = nz[q];   // nz ascending: i >= j
      L[i * n + j] += d * row[i] * row[j];
    }
    __syncwarp();
  }
  // middle-zone cones: A A' - W W' over the union of the cone rows' columns
#pragma unroll 1
  for (int k = 0; k < ncone; k++) {
    const int code = cones[-k], r = code & 0xffff, dim = code >> 16;
    int cnt = 0;
#pragma unroll 1
    for (int base = 0; base < n; base += 32) {
      const int c = base + lane;
      bool on = false;
      if (c < n)
        for (int a = 0; a < dim; a++) on = on || J[(r + a) * n + c] != 0.f;
      const unsigned bal = __ballot_sync(FULL_MASK, on);
      if (on) nz[cnt + __popc(bal & ((1u << lane) - 1u))] = c;
      cnt += __popc(bal);
    }
    __syncwarp();
    const int one[1] = {code};
    const int T = cnt * (cnt + 1) / 2;
#pragma unroll 1
    for (int t = lane; t < T; t += 32) {
      int p = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
      if ((p + 1) * (p + 2) / 2 <= t) p++;
      else if (p * (p + 1) / 2 > t) p--;
      const int q = t - p * (p + 1) / 2;
      const int i = nz[p], j = nz[q];
      L[i * n + j] += cone_entry(J, hau, ne, one, 1, n, i, j);
    }
    __syncwarp();
  }
  d_chol(L, n, n, lane, idiag, nz);
}

// ell: rows weigh with HD instead of D, plus the middle-zone cones
// inv = true (nv <= 32, no cones): L receives N = A^-1 instead of the factor
__device__ __forceinline__ void d_factor(Env& E, const int* act, int nact, const float* ddiag, float dscale, float* L, float* idiag,
                                         bool ell = false, const int* cones = nullptr, int ncone = 0, bool inv = false) {
  const DevModelDesc& m = *E.md;
  const int nv = m.nv, ne = m.nefc_max;
  const float* M = E.ws + m.w_M;
  const float* J = E.ws + m.w_J;
  const float* efc = E.ws + m.w_efc;
  const float* eD = efc + (ell ? EFC_HD : EFC_D) * ne;
  const float* hau = efc + EFC_HA * ne;
  if (nv > 64) d_factor_sparse(M, J, eD, act, nact, ddiag, dscale, nv, E.lane, reinterpret_cast<int*>(E.ws + m.w_nz), L, idiag, cones, ncone, hau, ne);
  else d_factor_smem(M, J, eD, act, nact, ddiag, dscale, nv, m.ldh, E.lane, L, idiag, cones, ncone, hau, ne, inv);
}

__device__ __noinline__ void impedance(const DevModelDesc& m, float sr0, float sr1, const float* si, float pos, float& k, float& b, float& imp) {
  float tc = sr0, dr = sr1;
  if (!(m.disableflags & (1 << 11)) && tc > 0 && tc < 2 * m.timestep) tc = 2 * m.timestep;
  float dmin = clampf(si[0], 1e-4f, 0.9999f), dmax = clampf(si[1], 1e-4f, 0.9999f);
  float width = fmaxf(si[2], 1e-12f), mid = clampf(si[3], 1e-4f, 0.9999f), power = fmaxf(si[4], 1.f);
  k = tc > 0 ? 1.f / (dmax * dmax * tc * tc * dr * dr) : -tc / (dmax * dmax);
  b = dr > 0 ? 2.f / (dmax * tc) : -dr / dmax;
  float x = fabsf(pos) / width;
  if (x >= 1.f) { imp = dmax; return; }
  float y = x < mid ? powf(x, power) / powf(mid, power - 1.f) : 1.f - powf(1.f - x, power) / powf(1.f - mid, power - 1.f);
  imp = clampf(dmin + y * (dmax - dmin), dmin, dmax);
}

__device__ __forceinline__ int rows_of(float dim) { int d = (int)dim; return d == 1 ? 1 : 2 * (d - 1); }

// Builds efc rows; returns nefc.  Row metadata: EFC_AREF (b during the
// build), EFC_D, EFC_FLOSS, EFC_TYPE, EFC_Y (k*imp*pos during the build),
// EFC_CON (contact index or -1).
// EXT: the extended kernel instance, which also builds elliptic contacts
// (reference model: MuJoCo's elliptic cone; normal row R_n = (1 - imp) / imp
// * invweight, friction rows R_j = R_n (mu_0 / mu_j)^2 / impratio, friction
// rows' aref without the position term).
template <bool EXT>
__device__ __noinline__ int d_constraints(Env& E, const StepParams& P, int ncon) {
  const DevModelDesc& m = *E.md;
  const bool ell = EXT && m.cone == 1;
  const int* it = E.it;
  const float* ft = E.ft;
  float* ws = E.ws;
  const int nv = m.nv;
  float* J = ws + m.w_J;
  float* efc = ws + m.w_efc;
  const int ne = m.nefc_max;
  const float* qpos = ws + m.w_qpos;
  const float* qvel = ws + m.w_qvel;
  float* con = ws + m.w_con;
  int nefc = 0;
  bool stop = false;
  if (m.disableflags & 1) return 0;
  // --- joint / tendon equality rows (static list): x1 = poly(x2) with
  // x = q - qpos0 for joints and length - length0 for fixed tendons
  // (reference: solver.hpp:259-289; bilateral rows, always in their
  // quadratic zone)
  if (!(m.disableflags & (1 << 1)) && m.neq > 0) {
    int nq_ = m.neq;
    if (nq_ > m.nefc_max) { nq_ = m.nefc_max; stop = true; }
    #pragma unroll 1
    for (int r = E.lane; r < nq_; r += 32) {
      const int* qi = it + m.i_eq + 5 * r;
      const bool ten = ldi(qi, 0) == 1;
      const int o1 = ldi(qi, 1), o2 = ldi(qi, 2);
      const float* f = ft + m.f_eq + 15 * r;
      float x1, v1, x2 = 0.f, v2 = 0.f;
      if (ten) {
        d_tendon_lv(m, ws, o1, x1, v1);
        if (o2 >= 0) d_tendon_lv(m, ws, o2, x2, v2);
      } else {
        x1 = qpos[ldi(qi, 3)];
        v1 = qvel[o1];
        if (o2 >= 0) { x2 = qpos[ldi(qi, 4)]; v2 = qvel[o2]; }
      }
      x1 -= ldf(f, 0);
      x2 -= ldf(f, 1);
      float poly = ldf(f, 2), dpoly = 0.f;
      if (o2 >= 0) {
        poly = ldf(f, 2) + x2 * (ldf(f, 3) + x2 * (ldf(f, 4) + x2 * (ldf(f, 5) + x2 * ldf(f, 6))));
        dpoly = ldf(f, 3) + x2 * (2.f * ldf(f, 4) + x2 * (3.f * ldf(f, 5) + x2 * 4.f * ldf(f, 6)));
      }
      const float pos = x1 - poly;
      const float vel = v1 - dpoly * v2;
      float si[5] = {ldf(f, 9), ldf(f, 10), ldf(f, 11), ldf(f, 12), ldf(f, 13)};
      float k, b, imp;
      impedance(m, ldf(f, 7), ldf(f, 8), si, pos, k, b, imp);
      const float R = fmaxf((1.f - imp) / imp * ldf(f, 14), 1e-15f);
      if (ten) {
        d_tendon_row(m, ws, o1, 1.f, J + r * nv);
        if (o2 >= 0) {
          const float* J2 = ws + m.w_ten + o2 * (nv + 2) + 2;
          #pragma unroll 1
          for (int c = 0; c < nv; c++) J[r * nv + c] -= dpoly * J2[c];
        }
      } else {
        #pragma unroll 1
        for (int c = 0; c < nv; c++) J[r * nv + c] = (c == o1 ? 1.f : 0.f) - (c == o2 ? dpoly : 0.f);
      }
      EfcRef e{efc + r, ne};
      e[EFC_D] = 1.f / R;
      e[EFC_AREF] = -b * vel - k * imp * pos;
      e[EFC_FLOSS] = 0;
      e[EFC_TYPE] = ROW_EQUALITY;
      e[EFC_CON] = -1;
    }
    nefc = nq_;
  }
  // --- frictionloss rows (static list)
  if (!stop && !(m.disableflags & (1 << 2)) && m.nfloss > 0) {
    const int r0 = nefc;
    int nf = m.nfloss;
    if (r0 + nf > m.nefc_max) { nf = m.nefc_max - r0; stop = true; }
    #pragma unroll 1
    for (int q = E.lane; q < nf; q += 32) {
      const int r = r0 + q;
      int dof = ldi(it, m.i_floss + q);
      const float* f = ft + m.f_floss + 8 * q;
      float si[5] = {ldf(f, 3), ldf(f, 4), ldf(f, 5), ldf(f, 6), ldf(f, 7)};
      float k, b, imp;
      impedance(m, ldf(f, 1), ldf(f, 2), si, 0.f, k, b, imp);
      float R = fmaxf((1.f - imp) / imp * ldf(ft, m.f_dof_invweight0 + dof), 1e-15f);
      #pragma unroll 1
      for (int c = 0; c < nv; c++) J[r * nv + c] = c == dof ? 1.f : 0.f;
      EfcRef e{efc + r, ne};
      e[EFC_D] = 1.f / R;
      e[EFC_AREF] = -b * qvel[dof];
      e[EFC_FLOSS] = ldf(f, 0);
      e[EFC_TYPE] = ROW_FRICTION;
      e[EFC_CON] = -1;
    }
    nefc = r0 + nf;
  }
  // --- tendon frictionloss rows after the dof ones (reference: solver.hpp:320-342)
  if (!stop && !(m.disableflags & (1 << 2)) && m.ntfloss > 0) {
    const int r0 = nefc;
    int nf = m.ntfloss;
    if (r0 + nf > m.nefc_max) { nf = m.nefc_max - r0; stop = true; }
    #pragma unroll 1
    for (int q = E.lane; q < nf; q += 32) {
      const int r = r0 + q;
      const int t = ldi(it, m.i_tfloss + q);
      const float* tf = ft + m.f_ten + MJB_TEN_FLOATS * t;
      float si[5] = {ldf(tf, TEN_SIFRI), ldf(tf, TEN_SIFRI + 1), ldf(tf, TEN_SIFRI + 2), ldf(tf, TEN_SIFRI + 3), ldf(tf, TEN_SIFRI + 4)};
      float k, b, imp, len, vel;
      impedance(m, ldf(tf, TEN_SRFRI), ldf(tf, TEN_SRFRI + 1), si, 0.f, k, b, imp);
      d_tendon_lv(m, ws, t, len, vel);
      const float R = fmaxf((1.f - imp) / imp * ldf(tf, TEN_INVW), 1e-15f);
      d_tendon_row(m, ws, t, 1.f, J + r * nv);
      EfcRef e{efc + r, ne};
      e[EFC_D] = 1.f / R;
      e[EFC_AREF] = -b * vel;
      e[EFC_FLOSS] = ldf(tf, TEN_FLOSS);
      e[EFC_TYPE] = ROW_FRICTION;
      e[EFC_CON] = -1;
    }
    nefc = r0 + nf;
  }
  // --- joint limit rows (lower then upper side, joint order)
  if (!stop && !(m.disableflags & (1 << 3))) {
    #pragma unroll 1
    for (int base = 0; base < m.nlimit; base += 32) {
      int li = base + E.lane;
      int act[2] = {0, 0};
      float dist[2] = {0, 0};
      if (li < m.nlimit) {
        int qa = ldi(it, m.i_limit + 3 * li + 2);
        const float* f = ft + m.f_limit + 10 * li;
        float q = qpos[qa];
        dist[0] = q - ldf(f, 0);
        dist[1] = ldf(f, 1) - q;
        float margin = ldf(f, 2);
        act[0] = dist[0] < margin;
        act[1] = dist[1] < margin;
      }
      int cnt = act[0] + act[1];
      int incl = warp_incl_scan(cnt, E.lane);
      int total = __shfl_sync(FULL_MASK, incl, 31);
      int r = nefc + incl - cnt;
      for (int s = 0; s < 2; s++) {
        if (!act[s]) continue;
        if (r >= m.nefc_max) break;
        int dof = ldi(it, m.i_limit + 3 * li + 1);
        const float* f = ft + m.f_limit + 10 * li;
        float si[5] = {ldf(f, 5), ldf(f, 6), ldf(f, 7), ldf(f, 8), ldf(f, 9)};
        float pos = dist[s] - ldf(f, 2), k, b, imp;
        impedance(m, ldf(f, 3), ldf(f, 4), si, pos, k, b, imp);
        float sg = s == 0 ? 1.f : -1.f;
        #pragma unroll 1
        for (int c = 0; c < nv; c++) J[r * nv + c] = c == dof ? sg : 0.f;
        float R = fmaxf((1.f - imp) / imp * ldf(ft, m.f_dof_invweight0 + dof), 1e-15f);
        EfcRef e{efc + r, ne};
        e[EFC_D] = 1.f / R;
        e[EFC_AREF] = -b * sg * qvel[dof] - k * imp * pos;
        e[EFC_FLOSS] = 0;
        e[EFC_TYPE] = ROW_LIMIT;
        e[EFC_CON] = -1;
        r++;
      }
      nefc += total;
      if (nefc > m.nefc_max) { nefc = m.nefc_max; stop = true; break; }
    }
    // --- tendon limit rows after the joint limits (reference: solver.hpp:370-395)
    #pragma unroll 1
    for (int base = 0; !stop && base < m.ntlimit; base += 32) {
      const int li = base + E.lane;
      int act[2] = {0, 0};
      float dist[2] = {0, 0}, len = 0.f, vel = 0.f;
      int t = 0;
      if (li < m.ntlimit) {
        t = ldi(it, m.i_tlimit + li);
        const float* tf = ft + m.f_ten + MJB_TEN_FLOATS * t;
        d_tendon_lv(m, ws, t, len, vel);
        dist[0] = len - ldf(tf, TEN_LO);
        dist[1] = ldf(tf, TEN_HI) - len;
        act[0] = dist[0] < ldf(tf, TEN_MARGIN);
        act[1] = dist[1] < ldf(tf, TEN_MARGIN);
      }
      const int cnt = act[0] + act[1];
      const int incl = warp_incl_scan(cnt, E.lane);
      const int total = __shfl_sync(FULL_MASK, incl, 31);
      int r = nefc + incl - cnt;
      for (int s = 0; s < 2; s++) {
        if (!act[s]) continue;
        if (r >= m.nefc_max) break;
        const float* tf = ft + m.f_ten + MJB_TEN_FLOATS * t;
        float si[5] = {ldf(tf, TEN_SILIM), ldf(tf, TEN_SILIM + 1), ldf(tf, TEN_SILIM + 2), ldf(tf, TEN_SILIM + 3), ldf(tf, TEN_SILIM + 4)};
        float pos = dist[s] - ldf(tf, TEN_MARGIN), k, b, imp;
        impedance(m, ldf(tf, TEN_SRLIM), ldf(tf, TEN_SRLIM + 1), si, pos, k, b, imp);
        const float sg = s == 0 ? 1.f : -1.f;
        d_tendon_row(m, ws, t, sg, J + r * nv);
        const float R = fmaxf((1.f - imp) / imp * ldf(tf, TEN_INVW), 1e-15f);
        EfcRef e{efc + r, ne};
        e[EFC_D] = 1.f / R;
        e[EFC_AREF] = -b * sg * vel - k * imp * pos;
        e[EFC_FLOSS] = 0;
        e[EFC_TYPE] = ROW_LIMIT;
        e[EFC_CON] = -1;
        r++;
      }
      nefc += total;
      if (nefc > m.nefc_max) { nefc = m.nefc_max; stop = true; }
    }
  }
  // --- contact rows: offsets by scan, then per-contact impedance, then J by dof lanes
  int row0 = nefc;
  if (!stop && !(m.disableflags & (1 << 4))) {
    #pragma unroll 1
    for (int base = 0; base < ncon; base += 32) {
      int c = base + E.lane;
      int nr = 0;
      float* cr = con + MJB_CONTACT_FLOATS * (c < ncon ? c : 0);
      if (c < ncon) nr = (cr[12] < cr[15]) ? (ell && cr[14] > 1.f ? (int)cr[14] : rows_of(cr[14])) : 0;
      int incl = warp_incl_scan(nr, E.lane);
      int total = __shfl_sync(FULL_MASK, incl, 31);
      int r0 = nefc + incl - nr;
      bool fits = r0 + nr <= m.nefc_max;
      unsigned bad = __ballot_sync(FULL_MASK, nr > 0 && !fits);
      if (bad) {
        // drop the first group that does not fit and every later contact
        int first = __ffs(bad) - 1;
        int keep_rows = __shfl_sync(FULL_MASK, r0, first) - nefc;
        if (c < ncon && E.lane >= first) nr = 0;
        total = keep_rows;
        stop = true;
      }
      if (c < ncon && nr > 0) {
        int p = (int)cr[13];
        const float* pf = ft + m.f_pair + 16 * p;
        float si[5] = {ldf(pf, 9), ldf(pf, 10), ldf(pf, 11), ldf(pf, 12), ldf(pf, 13)};
        float pos = cr[12] - cr[15], k, b, imp;
        impedance(m, ldf(pf, 7), ldf(pf, 8), si, pos, k, b, imp);
        float invw = ldf(pf, 14);
        int dim = (int)cr[14];
        float D;
        if (ell && dim > 1) {
          const float fs = P.rand_friction ? P.rand_friction[E.env] : 1.f;
          const float mu0 = ldf(pf, 2) * fs;
          const float Rn = fmaxf((1.f - imp) / imp * invw, 1e-15f);
          #pragma unroll 1
          for (int q = 0; q < nr; q++) {
            EfcRef e{efc + r0 + q, ne};
            e[EFC_AREF] = b;
            e[EFC_CON] = (float)c;
            if (q == 0) {
              e[EFC_D] = 1.f / Rn;
              e[EFC_Y] = k * imp * pos;
              e[EFC_FLOSS] = mu0 / sqrtf(m.impratio);
              e[EFC_TYPE] = ROW_ELLIPTIC;
            } else {
              const float mu = ldf(pf, 1 + q) * fs;
              e[EFC_D] = 1.f / fmaxf(Rn * (mu0 * mu0) / (mu * mu) / m.impratio, 1e-15f);
              e[EFC_Y] = 0.f;
              e[EFC_FLOSS] = mu;
              e[EFC_TYPE] = ROW_ELLFRIC;
            }
          }
        } else {
        if (dim == 1) {
          D = 1.f / fmaxf((1.f - imp) / imp * invw, 1e-15f);
        } else {
          float fs = P.rand_friction ? P.rand_friction[E.env] : 1.f;
          float mu0 = ldf(pf, 2) * fs;
          float Rf = fmaxf((1.f - imp) / imp * invw * (1.f + mu0 * mu0), 1e-15f);
          D = 1.f / fmaxf(2.f * mu0 * mu0 / m.impratio * Rf, 1e-15f);
        }
        #pragma unroll 1
        for (int q = 0; q < nr; q++) {
          EfcRef e{efc + r0 + q, ne};
          e[EFC_D] = D;
          e[EFC_AREF] = b;
          e[EFC_Y] = k * imp * pos;
          e[EFC_FLOSS] = 0;
          e[EFC_TYPE] = dim == 1 ? ROW_FRICTIONLESS : ROW_PYRAMID;
          e[EFC_CON] = (float)c;
        }
        }
      }
      nefc += total;
      if (stop) break;
    }
  }
  if (stop) env_status(E, MJB_STATUS_EFC_OVERFLOW);
  __syncwarp();
  // Jacobian rows of the contacts: one lane per dof
  if (nefc > row0) {
    const float* scom = ws + m.w_scom;
    const float* cdof = ws + m.w_cdof;
    #pragma unroll 1
    for (int i = E.lane; i < nv; i += 32) {
      int db = ldi(it, m.i_dof_bodyid + i);
      int dsub = ldi(it, m.i_body_subtreesize + db);
      const float* cd = cdof + 6 * i;
      int r = row0;
      #pragma unroll 1
      for (int c = 0; c < ncon && r < nefc; c++) {
        const float* cr = con + MJB_CONTACT_FLOATS * c;
        if (!(cr[12] < cr[15])) continue;
        int p = (int)cr[13];
        int b1 = ldi(it, m.i_pair + 6 * p + 2), b2 = ldi(it, m.i_pair + 6 * p + 3);
        float jp[3] = {0, 0, 0}, jr[3] = {0, 0, 0};
        for (int side = 0; side < 2; side++) {
          int body = side == 0 ? b2 : b1;
          if (!(db <= body && body < db + dsub)) continue;
          float sg = side == 0 ? 1.f : -1.f;
          int root = ldi(it, m.i_body_rootid + body);
          float off[3] = {cr[0] - scom[3 * root], cr[1] - scom[3 * root + 1], cr[2] - scom[3 * root + 2]}, x[3];
          cross3(cd, off, x);
          for (int a = 0; a < 3; a++) { jp[a] += sg * (cd[3 + a] + x[a]); jr[a] += sg * cd[a]; }
        }
        const float* fr = cr + 3;
        float jn = fr[0] * jp[0] + fr[1] * jp[1] + fr[2] * jp[2];
        int dim = (int)cr[14];
        if (dim == 1) {
          J[r * nv + i] = jn;
          r++;
          continue;
        }
        if (ell) {
          J[r * nv + i] = jn;
          #pragma unroll 1
          for (int dir = 0; dir < dim - 1; dir++) {
            const float* ax = (dir == 0 || dir == 3) ? fr + 3 : (dir == 1 || dir == 4) ? fr + 6 : fr;
            const float* src = dir < 2 ? jp : jr;
            J[(r + 1 + dir) * nv + i] = ax[0] * src[0] + ax[1] * src[1] + ax[2] * src[2];
          }
          r += dim;
          continue;
        }
        float fs = P.rand_friction ? P.rand_friction[E.env] : 1.f;
        const float* pf = ft + m.f_pair + 16 * p;
        #pragma unroll 1
        for (int dir = 0; dir < dim - 1; dir++) {
          const float* ax = (dir == 0 || dir == 3) ? fr + 3 : (dir == 1 || dir == 4) ? fr + 6 : fr;
          const float* src = dir < 2 ? jp : jr;
          float jt = ax[0] * src[0] + ax[1] * src[1] + ax[2] * src[2];
          float mu = ldf(pf, 2 + dir) * fs;
          J[r * nv + i] = jn + mu * jt;
          J[(r + 1) * nv + i] = jn - mu * jt;
          r += 2;
        }
      }
    }
    __syncwarp();
    // reference acceleration: aref = -b J v - k imp pos
    #pragma unroll 1
    for (int r = row0 + E.lane; r < nefc; r += 32) {
      float jv = dot_c(J + r * nv, qvel, nv);
      EfcRef e{efc + r, ne};
      e[EFC_AREF] = -e[EFC_AREF] * jv - e[EFC_Y];
    }
    __syncwarp();
  }
  return nefc;
}

// ------------------------------------------------------------ Newton solver
__device__ __forceinline__ bool row_quad(int type, float D, float fl, float y) {
  if (type == ROW_FRICTION) return fabsf(y) < fl / D;
  if (type == ROW_EQUALITY) return true;
  return y < 0.f;
}
__device__ __forceinline__ float row_force(int type, float D, float fl, float y) {
  if (type == ROW_FRICTION) return clampf(-D * y, -fl, fl);
  if (type == ROW_EQUALITY) return -D * y;
  return y < 0.f ? -D * y : 0.f;
}
__device__ __forceinline__ float row_cost(int type, float D, float fl, float y) {
  if (type == ROW_FRICTION) {
    float R = 1.f / D;
    if (fabsf(y) < fl * R) return 0.5f * D * y * y;
    return fl * fabsf(y) - 0.5f * fl * fl * R;
  }
  if (type == ROW_EQUALITY) return 0.5f * D * y * y;
  return y < 0.f ? 0.5f * D * y * y : 0.f;
}
__device__ __forceinline__ float row_cost_delta(int type, float D, float fl, float y, float dy) {
  bool q0 = row_quad(type, D, fl, y), q1 = row_quad(type, D, fl, y + dy);
  if (q0 && q1) return 0.5f * D * dy * (2.f * y + dy);
  if (type != ROW_FRICTION && !q0 && !q1) return 0.f;
  if (type == ROW_FRICTION && !q0 && !q1 && ((y > 0) == (y + dy > 0))) return fl * (fabsf(y + dy) - fabsf(y));
  return row_cost(type, D, fl, y + dy) - row_cost(type, D, fl, y);
}

// Elliptic contact group (MuJoCo's cone model; solver.hpp has pyramids
// only): jar y over the normal row and dim - 1 friction rows, fl[0] = mu,
// fl[j] = mu_j, U = (mu y_0, mu_j y_j), N = U_0, T = |U_t|.  Zones: top
// (N >= mu T) no force; bottom (mu N + T <= 0) every row quadratic with its
// own D; middle: cost 0.5 Dm (N - mu T)^2, Dm = D_0 / (mu^2 (1 + mu^2)).
// Returns the cost.  f (may be null): forces -ds/dy.  q (may be null):
// qhq = q' H q.  hd/ha/hu (may be null): the Hessian as row data, H = sum_j
// hd_j e_j e_j' + ha ha' - hu hu' (middle zone: hd_j = c mu_j^2 on the
// friction rows, ha = sqrt(Dm) grad(N - mu T), hu_j = sqrt(c) mu_j U_j / T,
// c = -Dm (N - mu T) mu / T > 0).  Arrays are indexed below 6 only.
__device__ __forceinline__ float cone_eval(int dim, const float* D, const float* fl, const float* y, const float* q, float* f, float& qhq,
                                           float* hd, float* ha, float* hu) {
  const float mu = fl[0];
  float U[6], T2 = 0.f;
  U[0] = mu * y[0];
#pragma unroll
  for (int j = 1; j < 6; j++) {
    U[j] = j < dim ? fl[j] * y[j] : 0.f;
    T2 += U[j] * U[j];
  }
  const float T = sqrtf(T2), N = U[0];
  float cost = 0.f;
  qhq = 0.f;
  if (N >= mu * T || (T <= 0.f && N >= 0.f)) {
#pragma unroll
    for (int j = 0; j < 6; j++)
      if (j < dim) {
        if (f) f[j] = 0.f;
        if (hd) { hd[j] = 0.f; ha[j] = 0.f; hu[j] = 0.f; }
      }
    return 0.f;
  }
  if (mu * N + T <= 0.f || (T <= 0.f && N < 0.f)) {
#pragma unroll
    for (int j = 0; j < 6; j++)
      if (j < dim) {
        if (f) f[j] = -D[j] * y[j];
        cost += 0.5f * D[j] * y[j] * y[j];
        if (q) qhq += D[j] * q[j] * q[j];
        if (hd) { hd[j] = D[j]; ha[j] = 0.f; hu[j] = 0.f; }
      }
    return cost;
  }
  const float Dm = D[0] / (mu * mu * (1.f + mu * mu)), NmT = N - mu * T, iT = 1.f / T;
  const float c = -Dm * NmT * mu * iT;
  cost = 0.5f * Dm * NmT * NmT;
  if (f) {
    f[0] = -Dm * NmT * mu;
#pragma unroll
    for (int j = 1; j < 6; j++)
      if (j < dim) f[j] = Dm * NmT * mu * U[j] * iT * fl[j];
  }
  if (q) {
    float aq = mu * q[0], wq = 0.f, sq = 0.f;
#pragma unroll
    for (int j = 1; j < 6; j++)
      if (j < dim) {
        const float w = fl[j] * U[j] * iT;
        aq -= mu * w * q[j];
        wq += w * q[j];
        sq += fl[j] * fl[j] * q[j] * q[j];
      }
    qhq = Dm * aq * aq + c * (sq - wq * wq);
  }
  if (hd) {
    const float sDm = sqrtf(Dm), sc = sqrtf(c);
    hd[0] = 0.f;
    ha[0] = sDm * mu;
    hu[0] = 0.f;
#pragma unroll
    for (int j = 1; j < 6; j++)
      if (j < dim) {
        const float w = fl[j] * U[j] * iT;
        hd[j] = c * fl[j] * fl[j];
        ha[j] = -sDm * mu * w;
        hu[j] = sc * w;
      }
  }
  return cost;
}

// rows of the elliptic group whose normal row is r (its contact's condim)
__device__ __forceinline__ int cone_dim(const Env& E, const float* efc, int ne, int r) {
  return (int)E.ws[E.md->w_con + MJB_CONTACT_FLOATS * (int)efc[EFC_CON * ne + r] + 14];
}

__device__ __forceinline__ void cone_load(const float* efc, int ne, int r, int dim, float* D, float* fl) {
#pragma unroll
  for (int j = 0; j < 6; j++)
    if (j < dim) {
      D[j] = efc[EFC_D * ne + r + j];
      fl[j] = efc[EFC_FLOSS * ne + r + j];
    }
}

// Cost of candidate x (Gauss term 0.5 d'M d with d = x - qacc_smooth, plus
// row costs).  `tmp` is nv floats of scratch.  Warp-uniform result.
template <bool EXT>
__device__ __noinline__ float d_cost(Env& E, int nefc, const float* x, float* tmp) {
  const DevModelDesc& m = *E.md;
  const int nv = m.nv, ne = m.nefc_max, lane = E.lane;
  const float* M = E.ws + m.w_M;
  const float* qas = E.ws + m.w_qas;
  const float* J = E.ws + m.w_J;
  const float* efc = E.ws + m.w_efc;
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) tmp[i] = x[i] - qas[i];
  __syncwarp();
  float c = 0;
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) c += 0.5f * tmp[i] * dot_c(M + i * nv, tmp, nv);
#pragma unroll 1
  for (int r = lane; r < nefc; r += 32) {
    const int ty = (int)efc[EFC_TYPE * ne + r];
    if (EXT && ty == ROW_ELLFRIC) continue;
    if (EXT && ty == ROW_ELLIPTIC) {
      const int dim = cone_dim(E, efc, ne, r);
      float D[6], fl[6], y[6], qhq;
#pragma unroll
      for (int j = 0; j < 6; j++)
        if (j < dim) y[j] = dot_c(J + (r + j) * nv, x, nv) - efc[EFC_AREF * ne + r + j];
      cone_load(efc, ne, r, dim, D, fl);
      c += cone_eval(dim, D, fl, y, nullptr, nullptr, qhq, nullptr, nullptr, nullptr);
      continue;
    }
    float y = dot_c(J + r * nv, x, nv) - efc[EFC_AREF * ne + r];
    c += row_cost(ty, efc[EFC_D * ne + r], efc[EFC_FLOSS * ne + r], y);
  }
  __syncwarp();
  return warp_sum(c);
}

// Forces (and the Hessian row data HD / HA / HU) from the jar in EFC_Y, for
// models with elliptic cones: the lane of a cone's normal row evaluates the
// whole group.
__device__ __noinline__ void d_forces_ell(Env& E, int nefc) {
  const DevModelDesc& m = *E.md;
  const int ne = m.nefc_max;
  float* efc = E.ws + m.w_efc;
#pragma unroll 1
  for (int r = E.lane; r < nefc; r += 32) {
    const int ty = (int)efc[EFC_TYPE * ne + r];
    if (ty == ROW_ELLFRIC) continue;
    if (ty == ROW_ELLIPTIC) {
      const int dim = cone_dim(E, efc, ne, r);
      float D[6], fl[6], y[6], qhq;
      cone_load(efc, ne, r, dim, D, fl);
#pragma unroll
      for (int j = 0; j < 6; j++)
        if (j < dim) y[j] = efc[EFC_Y * ne + r + j];
      // a group's rows are consecutive within each field: write in place
      cone_eval(dim, D, fl, y, nullptr, efc + EFC_FORCE * ne + r, qhq, efc + EFC_HD * ne + r, efc + EFC_HA * ne + r, efc + EFC_HU * ne + r);
      continue;
    }
    const float D = efc[EFC_D * ne + r], fl = efc[EFC_FLOSS * ne + r], y = efc[EFC_Y * ne + r];
    efc[EFC_FORCE * ne + r] = row_force(ty, D, fl, y);
    efc[EFC_HD * ne + r] = row_quad(ty, D, fl, y) ? D : 0.f;
  }
  __syncwarp();
}

// Line-search sums at step a along q = EFC_Q for elliptic models (per lane):
// g1 = -sum q' force(y + a q), g2 = sum q' H q; the cone groups are
// evaluated by their normal row's lane.
__device__ __noinline__ void ls_sums_ell(const Env& E, const float* efc, int ne, int nefc, float a, float& g1, float& g2) {
#pragma unroll 1
  for (int r = E.lane; r < nefc; r += 32) {
    const int ty = (int)efc[EFC_TYPE * ne + r];
    if (ty == ROW_ELLFRIC) continue;
    if (ty == ROW_ELLIPTIC) {
      const int dim = cone_dim(E, efc, ne, r);
      float D[6], fl[6], y[6], q[6], f[6], qhq;
      cone_load(efc, ne, r, dim, D, fl);
#pragma unroll
      for (int j = 0; j < 6; j++)
        if (j < dim) {
          q[j] = efc[EFC_Q * ne + r + j];
          y[j] = efc[EFC_Y * ne + r + j] + a * q[j];
        }
      cone_eval(dim, D, fl, y, q, f, qhq, nullptr, nullptr, nullptr);
#pragma unroll
      for (int j = 0; j < 6; j++)
        if (j < dim) g1 -= q[j] * f[j];
      g2 += qhq;
      continue;
    }
    const float q = efc[EFC_Q * ne + r], y = efc[EFC_Y * ne + r] + a * q, D = efc[EFC_D * ne + r], fl = efc[EFC_FLOSS * ne + r];
    g1 -= q * row_force(ty, D, fl, y);
    if (row_quad(ty, D, fl, y)) g2 += D * q * q;
  }
}

// Middle-zone cones (normal row with HA != 0) written downwards from
// cones[0] as normal row | dim << 16; returns their count.
__device__ __noinline__ int d_cone_list(const Env& E, int nefc, int* cones) {
  const DevModelDesc& m = *E.md;
  const int ne = m.nefc_max, lane = E.lane;
  const float* efc = E.ws + m.w_efc;
  int ncone = 0;
#pragma unroll 1
  for (int base = 0; base < nefc; base += 32) {
    const int r = base + lane;
    const bool cq = r < nefc && (int)efc[EFC_TYPE * ne + r] == ROW_ELLIPTIC && efc[EFC_HA * ne + r] != 0.f;
    const unsigned b = __ballot_sync(FULL_MASK, cq);
    if (cq) cones[-(ncone + __popc(b & ((1u << lane) - 1u)))] = r | (cone_dim(E, efc, ne, r) << 16);
    ncone += __popc(b);
  }
  __syncwarp();
  return ncone;
}

// Cost change of the rows along the step a q for elliptic models (per lane).
__device__ __noinline__ float cost_delta_ell(const Env& E, const float* efc, int ne, int nefc, float a) {
  float dc = 0.f;
#pragma unroll 1
  for (int r = E.lane; r < nefc; r += 32) {
    const int ty = (int)efc[EFC_TYPE * ne + r];
    if (ty == ROW_ELLFRIC) continue;
    if (ty == ROW_ELLIPTIC) {
      const int dim = cone_dim(E, efc, ne, r);
      float D[6], fl[6], y0[6], y1[6], qhq;
      cone_load(efc, ne, r, dim, D, fl);
#pragma unroll
      for (int j = 0; j < 6; j++)
        if (j < dim) {
          y0[j] = efc[EFC_Y * ne + r + j];
          y1[j] = y0[j] + a * efc[EFC_Q * ne + r + j];
        }
      dc += cone_eval(dim, D, fl, y1, nullptr, nullptr, qhq, nullptr, nullptr, nullptr) -
            cone_eval(dim, D, fl, y0, nullptr, nullptr, qhq, nullptr, nullptr, nullptr);
      continue;
    }
    dc += row_cost_delta(ty, efc[EFC_D * ne + r], efc[EFC_FLOSS * ne + r], efc[EFC_Y * ne + r], a * efc[EFC_Q * ne + r]);
  }
  return dc;
}

// g = Md - J'force; returns ||g||^2 and the magnitude of the summed terms
// (||Md||^2 + ||J'force||^2) that sets the FP32 round-off floor of g.
__device__ __forceinline__ float grad_update(const float* J, const float* force, const float* Md, float* grad, int nv, int nefc, int lane, float& terms) {
  float gn = 0, tn = 0;
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) {
    float f = dot_s(J + i, nv, force, nefc);
    float g = Md[i] - f;
    grad[i] = g;
    gn += g * g;
    tn += Md[i] * Md[i] + f * f;
  }
  terms = warp_sum(tn);
  return warp_sum(gn);
}

// Newton solve from the warm start; x (w_x) holds the result.  Returns the
// iteration count.  vec: Md, grad, p, Mp, tmp, -, -, -, idiag.
// The Hessian changes only when the set of rows in their quadratic zone
// does.  INV = true (for nv <= 32 without elliptic cones and nefc <= 128;
// the caller checks) keeps the inverse N = H^-1 instead of a factor, and
// updates it
// incrementally (MuJoCo's Newton solver keeps its factor incrementally the
// same way): rows that entered the set since the last rebuild are added and
// rows that left are removed by Sherman-Morrison rank-1 steps, as long as at
// most kMaxRank1 rows changed; more changes, or a removal that cancels,
// rebuild N from H by the sweep.  The direction is then p = -N g, one
// matrix-vector product instead of two triangular solves.  hm = true says
// H still holds M^-1 from the unconstrained solve, which then serves as
// the starting inverse (no active rows: no rebuild at all).
// Termination: improvement or gradient below tolerance * meaninertia * nv,
// where the gradient test also accepts the FP32 round-off floor of the
// gradient (16 eps times the norm of the terms it is summed from) -- below
// that floor FP32 cannot resolve it.
constexpr int kMaxRank1 = 32;

// Inverse mode of the Newton solver (nv <= 32, no elliptic cones, nefc <=
// 128): bring N = H^-1 in the H slot up to the rows now in their quadratic
// zone, then the direction p = -N grad (solver vectors 2 and 1).  The row-set words are in the sparse-index slot: words 0-3 the rows
// N includes, words 4-7 the rows active now.  have = false: N holds nothing
// usable (rebuild).  Otherwise up to kMaxRank1 changed rows go in by
// Sherman-Morrison (additions first), and more, or a cancelling removal,
// rebuild N from M and the listed active rows by the sweep.
__device__ __noinline__ void d_hinv_direction(Env& E, const int* act_list, int nact, bool have) {
  const DevModelDesc& m = *E.md;
  const int nv = m.nv, lane = E.lane;
  float* ws = E.ws;
  float* H = ws + m.w_H;
  float* hcol = H + nv * m.ldh;
  unsigned* wd = reinterpret_cast<unsigned*>(ws + m.w_nz);
  const float* J = ws + m.w_J;
  const float* eD = ws + m.w_efc + EFC_D * m.nefc_max;
  int nch = 0;
#pragma unroll
  for (int c = 0; c < 4; c++) nch += __popc(wd[c] ^ wd[4 + c]);
  bool full = !have || nch > kMaxRank1;
  if (!full && nch > 0) {
#pragma unroll 1
    for (int c = 0; c < 4; c++) {
      unsigned b = wd[4 + c] & ~wd[c];
      while (b) {
        const int r = 32 * c + __ffs(b) - 1;
        b &= b - 1;
        d_inv_rank1(H, nv, m.ldh, hcol, J + r * nv, sqrtf(eD[r]), 1.f, lane);
      }
    }
#pragma unroll 1
    for (int c = 0; c < 4 && !full; c++) {
      unsigned b = wd[c] & ~wd[4 + c];
      while (b && !full) {
        const int r = 32 * c + __ffs(b) - 1;
        b &= b - 1;
        full = !d_inv_rank1(H, nv, m.ldh, hcol, J + r * nv, sqrtf(eD[r]), -1.f, lane);
      }
    }
  }
  if (full) d_factor(E, act_list, nact, nullptr, 0.f, H, nullptr, false, nullptr, 0, true);
  __syncwarp();
  if (lane < 4) wd[lane] = wd[4 + lane];
  float* vec = ws + m.w_vec;
  const float pi = d_inv_apply(H, nv, m.ldh, hcol, vec + nv, lane);
  if (lane < nv) vec[2 * nv + lane] = -pi;
  __syncwarp();
}

template <bool EXT, bool INV>
__device__ __noinline__ int d_newton(Env& E, const StepParams& P, int nefc, int max_iter, const float* xpred, int& choice, bool hm) {
  (void)P;
  const DevModelDesc& m = *E.md;
  const bool ell = !INV && EXT && m.cone == 1;
  const int nv = m.nv, ne = m.nefc_max, lane = E.lane, ls_iter = m.ls_iterations;
  float* ws = E.ws;
  const float* M = ws + m.w_M;
  const float* qas = ws + m.w_qas;
  const float* J = ws + m.w_J;
  float* efc = ws + m.w_efc;
  float* H = ws + m.w_H;
  float* x = ws + m.w_x;
  int* act_list = reinterpret_cast<int*>(ws + m.w_active);
  const float* xw = ws + m.w_xwarm;
  float* vec = ws + m.w_vec;
  float *Md = vec, *grad = vec + nv, *p = vec + 2 * nv, *Mp = vec + 3 * nv, *tmp = vec + 4 * nv, *idiag = vec + 8 * nv;
  float* eY = efc + EFC_Y * ne;
  float* eF = efc + EFC_FORCE * ne;
  float* eQ = efc + EFC_Q * ne;
  const float* eD = efc + EFC_D * ne;
  const float* eA = efc + EFC_AREF * ne;
  const float* eL = efc + EFC_FLOSS * ne;
  const float* eT = efc + EFC_TYPE * ne;
  const float* eHD = efc + EFC_HD * ne;   // elliptic models only
  const float scale = m.scale, tol = m.tolerance;

  // warm start: lowest cost of smooth / previous / predicted
  choice = 0;
  const float* src = qas;
  if (!(m.disableflags & (1 << 8)) && nefc > 0) {
    float best = d_cost<EXT>(E, nefc, qas, tmp);
    float cw = d_cost<EXT>(E, nefc, xw, tmp);
    if (cw < best) { best = cw; choice = 1; }
    if (xpred) {
      float cp = d_cost<EXT>(E, nefc, xpred, tmp);
      if (cp <= best) { best = cp; choice = 2; }
    }
    src = choice == 1 ? xw : choice == 2 ? xpred : qas;
  }
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) {
    x[i] = src[i];
    tmp[i] = src[i] - qas[i];
  }
  __syncwarp();
  // state at x: d = x - a0, Md, y, force, grad
#pragma unroll 1
  for (int i = lane; i < nv; i += 32) Md[i] = dot_c(M + i * nv, tmp, nv);
#pragma unroll 1
  for (int r = lane; r < nefc; r += 32) {
    float y = dot_c(J + r * nv, x, nv) - eA[r];
    eY[r] = y;
    if (!ell) eF[r] = row_force((int)eT[r], eD[r], eL[r], y);
  }
  __syncwarp();
  if (ell) d_forces_ell(E, nefc);
  float terms;
  float gn = grad_update(J, eF, Md, grad, nv, nefc, lane, terms);
  __syncwarp();
  const float eps_floor = 16.f * 1.1920929e-7f;
  if (nefc == 0 || scale * sqrtf(gn) < tol || gn <= eps_floor * eps_floor * terms) return 0;
  int nact_prev = -1;
  int niter = 0;
  // inverse mode (INV: the caller checked nv <= 32, nefc <= 128, no
  // elliptic cones): the row-set words live in the sparse-index slot (words
  // 0-3: rows in N, 4-7: rows in their quadratic zone; bit r % 32 of word
  // r / 32), written by lane 0
  constexpr bool inc = INV;
  bool have = hm;
  if (inc && lane == 0)
    for (int c = 0; c < 8; c++) reinterpret_cast<unsigned*>(ws + m.w_nz)[c] = 0u;
#pragma unroll 1
  for (int iter = 0; iter < max_iter; iter++) {
    // compact list of rows in their quadratic zone (order preserved)
    int nact = 0;
    bool changed = false;
    if (inc && lane == 0)
      for (int c = 4; c < 8; c++) reinterpret_cast<unsigned*>(ws + m.w_nz)[c] = 0u;
#pragma unroll 1
    for (int base = 0; base < nefc; base += 32) {
      int r = base + lane;
      bool q = r < nefc && (ell ? eHD[r] > 0.f : row_quad((int)eT[r], eD[r], eL[r], eY[r]));
      unsigned b = __ballot_sync(FULL_MASK, q);
      if (inc && lane == 0) reinterpret_cast<unsigned*>(ws + m.w_nz)[4 + (base >> 5)] = b;
      int pos = nact + __popc(b & ((1u << lane) - 1u));
      if (q) {
        if (nact_prev < 0 || pos >= nact_prev || act_list[pos] != r) changed = true;
      }
      nact += __popc(b);
      changed = __any_sync(FULL_MASK, changed);
      __syncwarp();
      if (q) act_list[pos] = r;
    }
    if (nact != nact_prev) changed = true;
    __syncwarp();
    // middle-zone cones (their Hessian moves with y: refactor every
    // iteration while any is present), listed downwards from the end of the
    // active-row list: active rows + cones <= nefc, as a middle-zone cone's
    // normal row is not active
    int* cones = act_list + ne - 1;
    const int ncone = ell ? d_cone_list(E, nefc, cones) : 0;
    if (ncone) changed = true;
    if constexpr (INV) {
      d_hinv_direction(E, act_list, nact, have);
      have = true;
    } else {
      if (changed) {
        d_factor(E, act_list, nact, nullptr, 0.f, H, idiag, ell, cones, ncone);
        nact_prev = nact;
      }
#pragma unroll 1
      for (int i = lane; i < nv; i += 32) p[i] = -grad[i];
      __syncwarp();
      d_chol_solve(H, idiag, nv, m.ldh, p, lane);
    }
    // line-search coefficients A = p'Mp, B = p'Md, q = J p
    float A = 0, B = 0, gp = 0;
#pragma unroll 1
    for (int i = lane; i < nv; i += 32) {
      float s = dot_c(M + i * nv, p, nv);
      Mp[i] = s;
      A += p[i] * s;
      B += p[i] * Md[i];
      gp += grad[i] * p[i];
    }
#pragma unroll 1
    for (int r = lane; r < nefc; r += 32) eQ[r] = dot_c(J + r * nv, p, nv);
    A = warp_sum(A);
    B = warp_sum(B);
    gp = warp_sum(gp);
    __syncwarp();
    if (!(gp < 0.f)) break;
    // exact line search: safeguarded Newton on the monotone derivative
    float d0, h0;
    {
      float g1 = 0, g2 = 0;
      if (ell) ls_sums_ell(E, efc, ne, nefc, 0.f, g1, g2);
      else {
#pragma unroll 1
      for (int r = lane; r < nefc; r += 32) {
        int ty = (int)eT[r];
        float q = eQ[r], y = eY[r], D = eD[r], fl = eL[r];
        g1 -= q * row_force(ty, D, fl, y);
        if (row_quad(ty, D, fl, y)) g2 += D * q * q;
      }
      }
      d0 = B + warp_sum(g1);
      h0 = A + warp_sum(g2);
    }
    niter++;
    float alpha = 0;
    if (d0 < 0.f) {
      float lo = 0, dlo = d0, hi = -1, dhi = 0;
      float a = -d0 / h0;
#pragma unroll 1
      for (int it2 = 0; it2 < ls_iter; it2++) {
        float g1 = 0, g2 = 0;
        if (ell) ls_sums_ell(E, efc, ne, nefc, a, g1, g2);
        else {
#pragma unroll 1
        for (int r = lane; r < nefc; r += 32) {
          int ty = (int)eT[r];
          float q = eQ[r], y = eY[r] + a * q, D = eD[r], fl = eL[r];
          g1 -= q * row_force(ty, D, fl, y);
          if (row_quad(ty, D, fl, y)) g2 += D * q * q;
        }
        }
        float dd = a * A + B + warp_sum(g1);
        float hh = A + warp_sum(g2);
        if (dd < 0.f) { lo = a; dlo = dd; } else { hi = a; dhi = dd; }
        if (fabsf(dd) <= 1e-6f * fabsf(d0)) break;
        float an = a - dd / hh;
        if (hi >= 0.f && !(an > lo && an < hi)) {
          an = (dlo * hi - dhi * lo) / (dlo - dhi);
          if (!(an > lo && an < hi)) an = 0.5f * (lo + hi);
        }
        if (fabsf(an - a) <= 1e-6f * fabsf(a)) { a = an; break; }
        a = an;
      }
      alpha = a;
    }
    if (alpha == 0.f) break;
    // cost change along the step (accurate for small steps)
    float dc = 0;
    if (ell) dc = cost_delta_ell(E, efc, ne, nefc, alpha);
    else {
#pragma unroll 1
    for (int r = lane; r < nefc; r += 32) dc += row_cost_delta((int)eT[r], eD[r], eL[r], eY[r], alpha * eQ[r]);
    }
    dc = warp_sum(dc) + 0.5f * alpha * alpha * A + alpha * B;
    // update x, Md, y, force, grad
#pragma unroll 1
    for (int i = lane; i < nv; i += 32) {
      x[i] += alpha * p[i];
      Md[i] += alpha * Mp[i];
    }
#pragma unroll 1
    for (int r = lane; r < nefc; r += 32) {
      float y = eY[r] + alpha * eQ[r];
      eY[r] = y;
      if (!ell) eF[r] = row_force((int)eT[r], eD[r], eL[r], y);
    }
    __syncwarp();
    if (ell) d_forces_ell(E, nefc);
    gn = grad_update(J, eF, Md, grad, nv, nefc, lane, terms);
    __syncwarp();
    float improvement = -scale * dc;
    if (improvement < tol || scale * sqrtf(gn) < tol || gn <= eps_floor * eps_floor * terms) break;
  }
  return niter;
}

// qfrc_constraint = J' force into out
__device__ __noinline__ void d_jtf(Env& E, int nefc, float* out) {
  const DevModelDesc& m = *E.md;
  const int nv = m.nv, ne = m.nefc_max;
  const float* J = E.ws + m.w_J;
  const float* eF = E.ws + m.w_efc + EFC_FORCE * ne;
#pragma unroll 1
  for (int i = E.lane; i < nv; i += 32) out[i] = dot_s(J + i, nv, eF, nefc);
  __syncwarp();
}

// Semi-implicit Euler with optional implicit damping; returns false when the
// acceleration is not finite (caller resets the env).
__device__ __noinline__ void d_integrate(Env& E, const float* acc) {
  const DevModelDesc& m = *E.md;
  const int* it = E.it;
  float* ws = E.ws;
  float* qpos = ws + m.w_qpos;
  float* qvel = ws + m.w_qvel;
  const float h = m.timestep;
  #pragma unroll 1
  for (int i = E.lane; i < m.nv; i += 32) qvel[i] += h * acc[i];
  __syncwarp();
  #pragma unroll 1
  for (int j = E.lane; j < m.njnt; j += 32) {
    int qa = ldi(it, m.i_jnt_qposadr + j), da = ldi(it, m.i_jnt_dofadr + j), t = ldi(it, m.i_jnt_type + j);
    float* q = qpos + qa;
    const float* v = qvel + da;
    if (t == 2 || t == 3) { q[0] += h * v[0]; continue; }
    const float* w = v;
    float* qq = q;
    if (t == 0) {
      for (int k = 0; k < 3; k++) q[k] += h * v[k];
      w = v + 3;
      qq = q + 3;
    }
    float wn = sqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    float ha = 0.5f * h * wn;
    float sn, cs;
    sincosf(ha, &sn, &cs);
    float s = wn > 1e-12f ? sn / wn : 0.5f * h;
    float dq[4] = {cs, s * w[0], s * w[1], s * w[2]};
    float cur[4] = {qq[0], qq[1], qq[2], qq[3]}, nq[4];
    qmul(cur, dq, nq);
    qnormalize(nq);
    for (int k = 0; k < 4; k++) qq[k] = nq[k];
  }
  __syncwarp();
}

}  // namespace mjbdev
