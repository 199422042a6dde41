// Learned PP shell: a small MLP that predicts, from the local CIC density around a
// particle, the force that the cutoff-1 split (PM3 softened at 1 fine cell plus PP within
// 1 fine cell) misses against the cutoff-2 split of the plain kick.  No reference
// counterpart; oracle/mlp_oracle.py restates every step.
//
// Inputs of a particle at fine position x (periodic image of ng fine cells): log(1 + rho)
// of the CIC density of all particles on the 4^3 fine cells i0-1 .. i0+2 around
// i0 = floor(x - 0.5) (x fastest), then the offsets x - 0.5 - i0: 67 values, padded to 80.
// Network: 67 -> 128 -> 128 -> 128 -> 3, tanh-GELU, BF16 operands on the tensor cores
// (mma.sync m16n8k16, FP32 accumulation), FP32 biases and FP32 master weights for Adam.
//
// Kernels: positions per stored particle, the CIC density, the feature rows (training
// input), a generic C = A B^T GEMM with bias / GELU epilogue (training forward and
// backward, K a multiple of 16), GELU backward, column sums, transposes, the MSE loss,
// Adam, and the fused inference kernel of the kick: every warp takes 16 particles through
// all four layers with the weights resident in shared memory and adds the predicted force
// times the kick coefficient to vp of the interior particles.
#include <algorithm>
#include <cstdlib>

#include "common.cuh"

namespace cube {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------------------------
// positions, density, features

struct MlpPosK {
  int nt, nte, ncb, nnt, rcs, ng;
  int64_t ncells;  // extended coarse cells over all tiles
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *cell_base;
  float4 *pos;     // [n_used]: global fine position, w = 1 for interior copies
};

// one warp per extended coarse cell: fine position of every stored copy (kick.f90:292 decode,
// tile origin added, wrapped into the periodic image)
__global__ void __launch_bounds__(kWarps * 32) k_mlp_pos(MlpPosK p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t c = (int64_t)blockIdx.x * kWarps + warp;
  if (c >= p.ncells) return;
  const int64_t per = (int64_t)p.nte * p.nte * p.nte;
  const int t = (int)(c / per);
  const int64_t r = c - (int64_t)t * per;
  const int ci = (int)(r % p.nte), cj = (int)((r / p.nte) % p.nte), ck = (int)(r / ((int64_t)p.nte * p.nte));
  const int tx = t % p.nnt, ty = (t / p.nnt) % p.nnt, tz = t / (p.nnt * p.nnt);
  const int np = p.rhoc[c];
  const int64_t base = p.cell_base[c];
  const bool interior = ci >= p.ncb && ci < p.ncb + p.nt && cj >= p.ncb && cj < p.ncb + p.nt && ck >= p.ncb &&
                        ck < p.ncb + p.nt;
  const int cc[3] = {tx * p.nt + ci - p.ncb, ty * p.nt + cj - p.ncb, tz * p.nt + ck - p.ncb};
  for (int l = lane; l < np; l += 32) {
    const int16_t *q = p.xp + 3 * (base + l);
    float v[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double x = decode_pos(cc[d], q[d]) * p.rcs;
      x -= floor(x / p.ng) * p.ng;
      v[d] = (float)x;
      if (v[d] >= (float)p.ng) v[d] = 0.f;
    }
    p.pos[base + l] = make_float4(v[0], v[1], v[2], interior ? 1.f : 0.f);
  }
}

__device__ __forceinline__ int wrap_cell(int i, int ng) { return i < 0 ? i + ng : (i >= ng ? i - ng : i); }

// CIC density of the interior copies (each physical particle once) on the periodic fine grid
__global__ void k_mlp_cic(const float4 *pos, int64_t n, int ng, float *rho) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 q = pos[i];
    if (q.w == 0.f) continue;
    const float xs[3] = {q.x - 0.5f, q.y - 0.5f, q.z - 0.5f};
    int i0[3];
    float f[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float fl = floorf(xs[d]);
      i0[d] = (int)fl;
      f[d] = xs[d] - fl;
    }
#pragma unroll
    for (int dz = 0; dz < 2; dz++)
#pragma unroll
      for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
          const float w = (dx ? f[0] : 1.f - f[0]) * (dy ? f[1] : 1.f - f[1]) * (dz ? f[2] : 1.f - f[2]);
          const int64_t X = wrap_cell(i0[0] + dx, ng), Y = wrap_cell(i0[1] + dy, ng), Z = wrap_cell(i0[2] + dz, ng);
          atomicAdd(rho + (Z * ng + Y) * ng + X, w);
        }
  }
}

// the 67 inputs (padded to kMlpK1 with zeros) of the particle at q into out[0..kMlpK1); lrho holds
// log(1 + rho) per fine cell
__device__ __forceinline__ void mlp_inputs(float4 q, const float *__restrict__ rho, int ng, bf16 *out) {
  const float xs[3] = {q.x - 0.5f, q.y - 0.5f, q.z - 0.5f};
  int i0[3];
  float f[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const float fl = floorf(xs[d]);
    i0[d] = (int)fl;
    f[d] = xs[d] - fl;
  }
  int k = 0;
  for (int dz = -1; dz <= 2; dz++) {
    const int64_t Z = wrap_cell(wrap_cell(i0[2] + dz, ng), ng);
    for (int dy = -1; dy <= 2; dy++) {
      const int64_t Y = wrap_cell(wrap_cell(i0[1] + dy, ng), ng);
      const float *row = rho + (Z * ng + Y) * ng;
#pragma unroll
      for (int dx = -1; dx <= 2; dx++) out[k++] = __float2bfloat16_rn(__ldg(row + wrap_cell(i0[0] + dx, ng)));
    }
  }
  out[64] = __float2bfloat16_rn(f[0]);
  out[65] = __float2bfloat16_rn(f[1]);
  out[66] = __float2bfloat16_rn(f[2]);
  for (int j = kMlpIn; j < kMlpK1; j++) out[j] = __float2bfloat16_rn(0.f);
}

// feature rows X[i] for every stored copy (zeros for buffer copies)
__global__ void k_mlp_features(const float4 *pos, int64_t n, const float *rho, int ng, bf16 *X) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 q = pos[i];
    __align__(16) bf16 row[kMlpK1];
    if (q.w != 0.f) {
      mlp_inputs(q, rho, ng, row);
    } else {
      for (int j = 0; j < kMlpK1; j++) row[j] = __float2bfloat16_rn(0.f);
    }
    uint4 *dst = reinterpret_cast<uint4 *>(X + i * kMlpK1);
    const uint4 *src = reinterpret_cast<const uint4 *>(row);
#pragma unroll
    for (int j = 0; j < kMlpK1 / 8; j++) dst[j] = src[j];
  }
}

// ---------------------------------------------------------------------------------------------
// tensor-core helpers (mma.sync m16n8k16, BF16 in, FP32 accumulate)

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// tanh by the hardware approximation (tanh.approx.f32, relative error about 2^-11, below the
// BF16 rounding of the activations); training and inference use the same function
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// tanh-GELU, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), in five FP32 operations and one
// hardware tanh: the argument as z (c + c 0.044715 z^2), the result as 0.5 z + 0.5 z t
constexpr float kGeluC = 0.7978845608028654f, kGeluC3 = 0.7978845608028654f * 0.044715f;
__device__ __forceinline__ float gelu_tanh_arg(float z) { return z * fmaf(kGeluC3, z * z, kGeluC); }

__device__ __forceinline__ float gelu_f(float z) {
  const float t = tanh_hw(gelu_tanh_arg(z));
  const float hz = 0.5f * z;
  return fmaf(hz, t, hz);
}

__device__ __forceinline__ float gelu_grad_f(float z) {
  const float t = tanh_hw(gelu_tanh_arg(z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * 0.044715f * z * z);
}

__device__ __forceinline__ uint32_t ld_u32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// A fragment (16 x 16, rows row0.., k from k0) from a row-major bf16 tile with row stride ld
__device__ __forceinline__ void frag_a(uint32_t a[4], const bf16 *s, int ld, int row0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  a[0] = ld_u32(s + (row0 + g) * ld + k0 + 2 * t);
  a[1] = ld_u32(s + (row0 + g + 8) * ld + k0 + 2 * t);
  a[2] = ld_u32(s + (row0 + g) * ld + k0 + 2 * t + 8);
  a[3] = ld_u32(s + (row0 + g + 8) * ld + k0 + 2 * t + 8);
}

// B fragment (16 x 8, B(k, n) = W[n][k]) from a row-major [n][k] bf16 tile with row stride ld
__device__ __forceinline__ void frag_b(uint32_t b[2], const bf16 *s, int ld, int n0, int k0, int lane) {
  const int g = lane >> 2, t = lane & 3;
  b[0] = ld_u32(s + (n0 + g) * ld + k0 + 2 * t);
  b[1] = ld_u32(s + (n0 + g) * ld + k0 + 2 * t + 8);
}

// ---------------------------------------------------------------------------------------------
// generic GEMM: C[M][N] = A[M][K] B[N][K]^T + bias[N]; epilogue writes Z (FP32, pre-activation)
// and/or H = act(Z) (BF16).  64 x 64 tiles, 4 warps of 32 x 32, K steps of 16 staged in shared
// memory (rows padded to 24 bf16 against bank conflicts).  K % 16 == 0, lda % 8 == 0, ldb % 8 == 0.

constexpr int kGT = 64, kGK = 16, kGLd = 24;

__global__ void __launch_bounds__(128) k_gemm_nt(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B,
                                                 int ldb, int M, int N, int K, const float *__restrict__ bias,
                                                 float *Z, int ldz, bf16 *H, int ldh, int act) {
  __shared__ __align__(16) bf16 sa[kGT * kGLd], sb[kGT * kGLd];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  float acc[2][4][4] = {};
  const int lr = threadIdx.x >> 1, lc = (threadIdx.x & 1) * 8;  // staging: row, 8-element chunk
  for (int k0 = 0; k0 < K; k0 += kGK) {
    uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
    if (m0 + lr < M) va = *reinterpret_cast<const uint4 *>(A + (int64_t)(m0 + lr) * lda + k0 + lc);
    if (n0 + lr < N) vb = *reinterpret_cast<const uint4 *>(B + (int64_t)(n0 + lr) * ldb + k0 + lc);
    *reinterpret_cast<uint4 *>(sa + lr * kGLd + lc) = va;
    *reinterpret_cast<uint4 *>(sb + lr * kGLd + lc) = vb;
    __syncthreads();
    uint32_t fa[2][4], fb[4][2];
#pragma unroll
    for (int i = 0; i < 2; i++) frag_a(fa[i], sa, kGLd, wm * 32 + i * 16, 0, lane);
#pragma unroll
    for (int j = 0; j < 4; j++) frag_b(fb[j], sb, kGLd, wn * 32 + j * 8, 0, lane);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], fa[i], fb[j]);
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int r = m0 + wm * 32 + i * 16 + g + (e >> 1) * 8;
        const int c = n0 + wn * 32 + j * 8 + 2 * t + (e & 1);
        if (r >= M || c >= N) continue;
        const float z = acc[i][j][e] + (bias ? bias[c] : 0.f);
        if (Z) Z[(int64_t)r * ldz + c] = z;
        if (H) H[(int64_t)r * ldh + c] = __float2bfloat16_rn(act ? gelu_f(z) : z);
      }
}

// ---------------------------------------------------------------------------------------------
// training elementwise kernels

// dZ = dA * gelu'(Z) for the [rows][n] block; FP32 and BF16 copies
__global__ void k_gelu_bwd(const float *da, const float *z, int64_t count, float *dz, bf16 *dzb) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = da[i] * gelu_grad_f(z[i]);
    dz[i] = v;
    dzb[i] = __float2bfloat16_rn(v);
  }
}

// out[c] = sum_r in[r][c] over rows (one block per 32 columns, FP64 partials)
__global__ void k_colsum(const float *in, int rows, int cols, int ncols_out, float *out) {
  __shared__ double part[8][32];
  const int c = blockIdx.x * 32 + (threadIdx.x & 31), w = threadIdx.x >> 5;
  double s = 0.0;
  if (c < cols)
    for (int r = w; r < rows; r += 8) s += in[(int64_t)r * cols + c];
  part[w][threadIdx.x & 31] = s;
  __syncthreads();
  if (w == 0 && c < ncols_out) {
    double t = 0.0;
    for (int k = 0; k < 8; k++) t += part[k][threadIdx.x];
    out[c] = (float)t;
  }
}

// out[C][R] = in[R][C] (bf16), 32 x 32 tiles
__global__ void k_transpose_bf16(const bf16 *in, int R, int C, bf16 *out) {
  __shared__ bf16 tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < R && c < C) ? in[(int64_t)r * C + c] : __float2bfloat16_rn(0.f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(int64_t)c * R + r] = tile[threadIdx.x][k];
  }
}

// dY = 2 (Y - T) / (rows * 3) in the first 3 of kMlpOutPad columns (rest 0), and the mean loss
__global__ void k_mse(const float *y, const float *t, int rows, float *dy, bf16 *dyb, float *loss) {
  float s = 0.f;
  const float sc = 2.0f / (3.0f * rows);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * kMlpOutPad; i += gridDim.x * blockDim.x) {
    const int r = i / kMlpOutPad, c = i % kMlpOutPad;
    float d = 0.f;
    if (c < kMlpOut) {
      const float e = y[i] - t[r * kMlpOut + c];
      s += e * e;
      d = sc * e;
    }
    dy[i] = d;
    dyb[i] = __float2bfloat16_rn(d);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (3.0f * rows));
}

// gather training rows: xb[r] = X[rows[r]], tb[r] = T[rows[r]]
__global__ void k_mlp_gather(const bf16 *X, const float *T, const int32_t *rows, int n, bf16 *xb, float *tb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * (kMlpK1 / 8); i += gridDim.x * blockDim.x) {
    const int r = i / (kMlpK1 / 8), j = i % (kMlpK1 / 8);
    const int64_t src = rows[r];
    reinterpret_cast<uint4 *>(xb + (int64_t)r * kMlpK1)[j] = reinterpret_cast<const uint4 *>(X + src * kMlpK1)[j];
    if (j < kMlpOut) tb[r * kMlpOut + j] = T[src * kMlpOut + j];
  }
}

// Adam on the FP32 master parameters, then the BF16 weight copies and their transposes
__global__ void k_adam(float *w, const float *grad, float *m, float *v, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 weights wb (layer l: [Np][K], W4 padded to kMlpOutPad rows) and transposes wt ([K][Np])
__global__ void k_mlp_pack(const float *master, bf16 *wb, bf16 *wt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpWbElems; i += gridDim.x * blockDim.x) {
    int l = 0;
    while (l < 3 && i >= mlp_wboff(l + 1)) l++;
    const int K = mlp_K(l), Np = mlp_Np(l), N = mlp_N(l);
    const int e = i - mlp_wboff(l), n = e / K, k = e % K;
    const float v = n < N ? master[mlp_woff(l) + n * K + k] : 0.f;
    const bf16 b = __float2bfloat16_rn(v);
    wb[i] = b;
    wt[mlp_wboff(l) + k * Np + n] = b;
  }
}

// ---------------------------------------------------------------------------------------------
// fused inference + kick

constexpr int kLd1 = kMlpK1 + 8, kLdW = kMlpW + 8;  // padded smem row strides (bf16)
constexpr int kApplyWarps = 10;                     // 94 KB of weights + 11.5 KB per warp
constexpr size_t kApplySmem = sizeof(bf16) * ((size_t)kMlpW * kLd1 + 2 * (size_t)kMlpW * kLdW + 8 * (size_t)kLdW) +
                              sizeof(float) * (3 * kMlpW + 8) +
                              sizeof(bf16) * (size_t)kApplyWarps * 16 * (kLd1 + 2 * kLdW);

struct MlpApplyK {
  const bf16 *wb;
  const float *master;
  const float4 *pos;
  const float *rho;
  int ng;
  int64_t n;
  float *vp;
  float coef;  // kick coefficient times the output scale
};

// copy one layer [Np][K] from global to shared rows of stride ld
__device__ __forceinline__ void load_layer(bf16 *dst, int ld, const bf16 *src, int Np, int K) {
  for (int i = threadIdx.x; i < Np * (K / 8); i += blockDim.x) {
    const int n = i / (K / 8), c = (i % (K / 8)) * 8;
    *reinterpret_cast<uint4 *>(dst + n * ld + c) = *reinterpret_cast<const uint4 *>(src + n * K + c);
  }
}

// one hidden layer for the warp's 16 rows: out = gelu(in W^T + b), in [16][K] (stride ldi)
template <int K>
__device__ __forceinline__ void warp_layer(const bf16 *in, int ldi, const bf16 *W, int ldw, const float *b,
                                           bf16 *out, int ldo, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
  for (int nh = 0; nh < kMlpW; nh += 64) {  // two halves of 64 outputs keep the accumulators small
    float acc[8][4] = {};
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
      uint32_t a[4];
      frag_a(a, in, ldi, 0, k0, lane);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        uint32_t bb[2];
        frag_b(bb, W, ldw, nh + j * 8, k0, lane);
        mma_bf16(acc[j], a, bb);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = nh + j * 8 + 2 * t;
      const float b0 = b[c], b1 = b[c + 1];
      *reinterpret_cast<__nv_bfloat162 *>(out + g * ldo + c) =
          __floats2bfloat162_rn(gelu_f(acc[j][0] + b0), gelu_f(acc[j][1] + b1));
      *reinterpret_cast<__nv_bfloat162 *>(out + (g + 8) * ldo + c) =
          __floats2bfloat162_rn(gelu_f(acc[j][2] + b0), gelu_f(acc[j][3] + b1));
    }
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kApplyWarps * 32, 1) k_mlp_apply(MlpApplyK p) {
  extern __shared__ __align__(16) unsigned char mlp_smem[];
  bf16 *w1 = reinterpret_cast<bf16 *>(mlp_smem);
  bf16 *w2 = w1 + kMlpW * kLd1;
  bf16 *w3 = w2 + kMlpW * kLdW;
  bf16 *w4 = w3 + kMlpW * kLdW;
  float *bias = reinterpret_cast<float *>(w4 + 8 * kLdW);  // b1 b2 b3 [128] each, b4 [8]
  bf16 *act = reinterpret_cast<bf16 *>(bias + 3 * kMlpW + 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bf16 *xs = act + warp * 16 * (kLd1 + 2 * kLdW);
  bf16 *ha = xs + 16 * kLd1, *hb = ha + 16 * kLdW;

  load_layer(w1, kLd1, p.wb + mlp_wboff(0), kMlpW, kMlpK1);
  load_layer(w2, kLdW, p.wb + mlp_wboff(1), kMlpW, kMlpW);
  load_layer(w3, kLdW, p.wb + mlp_wboff(2), kMlpW, kMlpW);
  load_layer(w4, kLdW, p.wb + mlp_wboff(3), 8, kMlpW);
  for (int i = threadIdx.x; i < 3 * kMlpW + 8; i += blockDim.x) {
    float v = 0.f;
    if (i < 3 * kMlpW) v = p.master[mlp_boff(i / kMlpW) + i % kMlpW];
    else if (i - 3 * kMlpW < kMlpOut) v = p.master[mlp_boff(3) + i - 3 * kMlpW];
    bias[i] = v;
  }
  __syncthreads();

  const int g = lane >> 2, t = lane & 3;
  const int64_t ntiles = (p.n + 15) / 16;
  for (int64_t tile = (int64_t)blockIdx.x * kApplyWarps + warp; tile < ntiles;
       tile += (int64_t)gridDim.x * kApplyWarps) {
    const int64_t r0 = tile * 16;
    // inputs of the 16 rows: two lanes per row, 40 inputs each
    {
      const int rr = lane >> 1, half = lane & 1;
      const int64_t i = r0 + rr;
      __align__(16) bf16 row[kMlpK1];
      const float4 q = i < p.n ? p.pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      if (i < p.n && q.w != 0.f) {
        mlp_inputs(q, p.rho, p.ng, row);
      } else {
        for (int j = 0; j < kMlpK1; j++) row[j] = __float2bfloat16_rn(0.f);
      }
      for (int j = half * 40; j < half * 40 + 40; j += 8)
        *reinterpret_cast<uint4 *>(xs + rr * kLd1 + j) = *reinterpret_cast<const uint4 *>(row + j);
    }
    __syncwarp();
    warp_layer<kMlpK1>(xs, kLd1, w1, kLd1, bias, ha, kLdW, lane);
    warp_layer<kMlpW>(ha, kLdW, w2, kLdW, bias + kMlpW, hb, kLdW, lane);
    warp_layer<kMlpW>(hb, kLdW, w3, kLdW, bias + 2 * kMlpW, ha, kLdW, lane);
    // output layer: one n8 tile (outputs 0..2 are used)
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k0 = 0; k0 < kMlpW; k0 += 16) {
      uint32_t a[4], bb[2];
      frag_a(a, ha, kLdW, 0, k0, lane);
      frag_b(bb, w4, kLdW, 0, k0, lane);
      mma_bf16(acc, a, bb);
    }
    // lanes with t = 0 hold outputs 0, 1 and t = 1 holds output 2 of rows g and g + 8
    if (t < 2) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int64_t i = r0 + g + 8 * h;
        if (i >= p.n || p.pos[i].w == 0.f) continue;
        float *v = p.vp + 3 * i + 2 * t;
        v[0] += p.coef * (acc[2 * h] + bias[3 * kMlpW + 2 * t]);
        if (t == 0) v[1] += p.coef * (acc[2 * h + 1] + bias[3 * kMlpW + 1]);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------------
// fused inference + kick on the 5th-generation tensor cores (tcgen05): 128 particles per tile,
// accumulators in tensor memory
//
// Two warpgroups per CTA, one CTA per SM, each warpgroup with its own tile: while one runs its
// epilogue (features, or bias + GELU + BF16 of a layer), the other's MMAs run.  A thread owns
// one particle (row m = thread index in the warpgroup = TMEM lane).  The operands sit in shared
// memory in the K-major layout without swizzle that the UMMA descriptors read: core matrices
// of 8 rows x 16 bytes, stored chunk-major, element (r, k) of an R-row matrix at byte
//   ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so one MMA step of K = 16 covers two 8-element chunks (leading-byte offset (R / 8) * 128 between
// them, stride-byte offset 128 between 8-row groups).  Layer l: D[128][N] = A[128][K] W_l^T with
// A the warpgroup's activation buffer and W_l [N][K] (N = 128, or 16 for the output layer), issued
// by one thread as K / 16 tcgen05.mma and one tcgen05.commit to the warpgroup's mbarrier.

constexpr int kTcRows = 128;                // particles per tile (UMMA M)
constexpr int kTcGroups = 4;                // warpgroups per CTA, each with its own tile
constexpr int kTcThreads = kTcGroups * kTcRows;
constexpr size_t kTcW1 = (size_t)kMlpW * kMlpK1 * 2, kTcW = (size_t)kMlpW * kMlpW * 2,
                 kTcW4 = (size_t)kMlpOutPad * kMlpW * 2;
constexpr size_t kTcAct = (size_t)kTcRows * kMlpW * 2;  // one warpgroup's activations
constexpr size_t kTcOffW2 = kTcW1, kTcOffW3 = kTcOffW2 + kTcW, kTcOffW4 = kTcOffW3 + kTcW,
                 kTcOffAct = kTcOffW4 + kTcW4, kTcOffBias = kTcOffAct + kTcGroups * kTcAct,
                 kTcOffBar = kTcOffBias + sizeof(float) * (3 * kMlpW + kMlpOutPad),
                 kTcSmem = kTcOffBar + 8 * kTcGroups + 16;
constexpr uint32_t kTcCols = 128 * kTcGroups;  // TMEM columns: 128 per warpgroup
constexpr unsigned long long kTcWaitNs = 1000000000ull;  // bound of one mbarrier wait: 1 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, k) of an R-row operand in the chunk-major core-matrix layout
__device__ __forceinline__ uint32_t umma_off(int r, int k, int R) {
  return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: K-major, no swizzle; start, leading and stride byte
// offsets in 16-byte units, version 1 (bits 46-47)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 A and B (K-major), FP32 accumulator, M = 128, N
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void wg_sync(int wg) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(kTcRows) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait for the phase of an mbarrier to complete, for at most kTcWaitNs; false on a timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > kTcWaitNs) return false;
  }
}

// every thread of the warpgroup gets the AND of v over the warpgroup (also a warpgroup barrier)
__device__ __forceinline__ bool wg_all(int wg, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + wg), "r"(kTcRows)
      : "memory");
  return r != 0;
}

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float v[4]) {
  uint32_t r[4];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 4; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// the inputs of mlp_inputs written straight into row m of the activation buffer, one 8-value
// chunk at a time: chunk 2 dz + h holds the stencil rows dy = 2h - 1, 2h of plane dz (x fastest),
// chunk 8 the offsets, chunk 9 zeros
__device__ __forceinline__ void tc_inputs(float4 q, bool live, const float *__restrict__ rho, int ng,
                                          unsigned char *act, int m) {
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  if (!live) {
#pragma unroll
    for (int c = 0; c < kMlpK1 / 8; c++) *reinterpret_cast<uint4 *>(act + umma_off(m, 8 * c, kTcRows)) = zero;
    return;
  }
  const float xs[3] = {q.x - 0.5f, q.y - 0.5f, q.z - 0.5f};
  int i0[3];
  float f[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const float fl = floorf(xs[d]);
    i0[d] = (int)fl;
    f[d] = xs[d] - fl;
  }
  int X[4];
#pragma unroll
  for (int dx = 0; dx < 4; dx++) X[dx] = wrap_cell(i0[0] + dx - 1, ng);
#pragma unroll 1
  for (int c = 0; c < 8; c++) {
    const int dz = c >> 1, h = c & 1;
    const int64_t Z = wrap_cell(wrap_cell(i0[2] + dz - 1, ng), ng);
    __align__(16) __nv_bfloat162 v[4];
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int64_t Y = wrap_cell(wrap_cell(i0[1] + 2 * h + r - 1, ng), ng);
      const float *row = rho + (Z * ng + Y) * ng;
      v[2 * r] = __floats2bfloat162_rn(__ldg(row + X[0]), __ldg(row + X[1]));
      v[2 * r + 1] = __floats2bfloat162_rn(__ldg(row + X[2]), __ldg(row + X[3]));
    }
    *reinterpret_cast<uint4 *>(act + umma_off(m, 8 * c, kTcRows)) = *reinterpret_cast<const uint4 *>(v);
  }
  __align__(16) __nv_bfloat162 o[4];
  o[0] = __floats2bfloat162_rn(f[0], f[1]);
  o[1] = __floats2bfloat162_rn(f[2], 0.f);
  o[2] = o[3] = __floats2bfloat162_rn(0.f, 0.f);
  *reinterpret_cast<uint4 *>(act + umma_off(m, 64, kTcRows)) = *reinterpret_cast<const uint4 *>(o);
  *reinterpret_cast<uint4 *>(act + umma_off(m, 72, kTcRows)) = zero;
}

// copy layer l ([R][K] row-major in global) into the chunk-major layout
__device__ __forceinline__ void tc_load_layer(unsigned char *dst, const bf16 *src, int R, int K) {
  for (int i = threadIdx.x; i < R * (K / 8); i += blockDim.x) {
    const int r = i / (K / 8), c = i % (K / 8);
    *reinterpret_cast<uint4 *>(dst + umma_off(r, 8 * c, R)) = *reinterpret_cast<const uint4 *>(src + r * K + 8 * c);
  }
}

// issue one layer: D (TMEM) = A W^T over K / 16 steps, then commit to the mbarrier
__device__ __forceinline__ void tc_issue(uint32_t tmem_d, uint32_t a_base, uint32_t w_base, int K, int N,
                                         uint32_t bar) {
  const uint32_t lbo_a = (kTcRows / 8) * 128, lbo_w = (uint32_t)(N / 8) * 128;
  const uint32_t idesc = umma_idesc(N);
  for (int s = 0; s < K / 16; s++) {
    const uint64_t ad = umma_desc(a_base + 2 * s * lbo_a, lbo_a, 128);
    const uint64_t bd = umma_desc(w_base + 2 * s * lbo_w, lbo_w, 128);
    umma_bf16(tmem_d, ad, bd, idesc, s > 0 ? 1u : 0u);
  }
  umma_commit(bar);
}

__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_apply_tc(MlpApplyK p, int32_t *err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char *w1 = tc_smem, *w2 = tc_smem + kTcOffW2, *w3 = tc_smem + kTcOffW3, *w4 = tc_smem + kTcOffW4;
  float *bias = reinterpret_cast<float *>(tc_smem + kTcOffBias);  // b1 b2 b3 [128] each, b4 [16]
  uint64_t *bars = reinterpret_cast<uint64_t *>(tc_smem + kTcOffBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tc_smem + kTcOffBar + 8 * kTcGroups);
  const int tid = threadIdx.x, wg = tid / kTcRows, m = tid % kTcRows, warp = tid >> 5;
  unsigned char *act = tc_smem + kTcOffAct + wg * kTcAct;

  tc_load_layer(w1, p.wb + mlp_wboff(0), kMlpW, kMlpK1);
  tc_load_layer(w2, p.wb + mlp_wboff(1), kMlpW, kMlpW);
  tc_load_layer(w3, p.wb + mlp_wboff(2), kMlpW, kMlpW);
  tc_load_layer(w4, p.wb + mlp_wboff(3), kMlpOutPad, kMlpW);
  for (int i = tid; i < 3 * kMlpW + kMlpOutPad; i += blockDim.x) {
    float v = 0.f;
    if (i < 3 * kMlpW) v = p.master[mlp_boff(i / kMlpW) + i % kMlpW];
    else if (i - 3 * kMlpW < kMlpOut) v = p.master[mlp_boff(3) + i - 3 * kMlpW];
    bias[i] = v;
  }
  if (tid == 0) {
    for (int b = 0; b < kTcGroups; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();  // the weights were written by ordinary stores; the tensor cores read them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot + (uint32_t)(wg * kMlpW);  // this warpgroup's 128 columns
  const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;  // TMEM lanes of this warp
  const uint32_t bar = smem_u32(&bars[wg]);
  const uint32_t a_s = smem_u32(act), w1_s = smem_u32(w1), w2_s = smem_u32(w2), w3_s = smem_u32(w3),
                 w4_s = smem_u32(w4);
  uint32_t phase = 0;
  bool ok = true;

  const int64_t ntiles = (p.n + kTcRows - 1) / kTcRows;
  for (int64_t tile = (int64_t)blockIdx.x * kTcGroups + wg; tile < ntiles && ok;
       tile += (int64_t)gridDim.x * kTcGroups) {
    const int64_t i = tile * kTcRows + m;
    const float4 q = i < p.n ? p.pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool live = i < p.n && q.w != 0.f;
    tc_inputs(q, live, p.rho, p.ng, act, m);  // layer-1 input row of this particle
    // layers 1-3 (N = 128): MMA, then bias + GELU + BF16 back into the activation buffer
#pragma unroll 1
    for (int l = 0; l < 3 && ok; l++) {
      fence_async_smem();
      tc_fence_before();
      wg_sync(wg);
      if (m == 0) {
        tc_fence_after();
        tc_issue(tmem, a_s, l == 0 ? w1_s : (l == 1 ? w2_s : w3_s), l == 0 ? kMlpK1 : kMlpW, kMlpW, bar);
      }
      ok = wg_all(wg, mbar_wait(bar, phase));
      phase ^= 1u;
      tc_fence_after();
      if (!ok) break;
      const float *b = bias + l * kMlpW;
#pragma unroll 1
      for (int c0 = 0; c0 < kMlpW; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + lane_base + (uint32_t)c0, v);
        __align__(16) __nv_bfloat162 h[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
          h[j] = __floats2bfloat162_rn(gelu_f(v[2 * j] + b[c0 + 2 * j]), gelu_f(v[2 * j + 1] + b[c0 + 2 * j + 1]));
#pragma unroll
        for (int c = 0; c < 2; c++)
          *reinterpret_cast<uint4 *>(act + umma_off(m, c0 + 8 * c, kTcRows)) = reinterpret_cast<const uint4 *>(h)[c];
      }
    }
    if (!ok) break;
    // output layer (N = 16, outputs 0..2 used) and the kick
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    if (m == 0) {
      tc_fence_after();
      tc_issue(tmem, a_s, w4_s, kMlpW, kMlpOutPad, bar);
    }
    ok = wg_all(wg, mbar_wait(bar, phase));
    phase ^= 1u;
    tc_fence_after();
    if (!ok) break;
    float y[4];
    tmem_ld4(tmem + lane_base, y);
    if (live) {
      float *v = p.vp + 3 * i;
      v[0] += p.coef * (y[0] + bias[3 * kMlpW + 0]);
      v[1] += p.coef * (y[1] + bias[3 * kMlpW + 1]);
      v[2] += p.coef * (y[2] + bias[3 * kMlpW + 2]);
    }
    tc_fence_before();  // the next tile's MMA overwrites these columns
  }
  if (!ok) {
    // a wait gave up while this warpgroup's MMA may still run: wait once more (also bounded) for
    // its commit before the tensor memory is released
    if (m == 0) atomicOr(err, 1 << CUBE_ERR_TIMEOUT);
    (void)mbar_wait(bar, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kTcCols));
  }
}

// ---------------------------------------------------------------------------------------------
// training GEMM on the 5th-generation tensor cores: C[M][N] = A[M][K] B[N][K]^T + bias[N] with the
// epilogue of k_gemm_nt (Z in FP32, H = act(Z) in BF16).  One warpgroup per CTA and a 128-row tile
// of C (UMMA M = 128, one TMEM lane per row); the CTA's N columns (a multiple of 16, at most 128)
// accumulate in TMEM.  K advances 64 at a time through two shared-memory stages: the loads of a
// stage (cp.async, 16 bytes, into the K-major core-matrix layout) overlap the MMAs of the other,
// whose tcgen05.commit to the stage's mbarrier frees it.  Rows of A past M and of B past N are
// zero-filled.  K % 16 == 0, lda % 8 == 0, ldb % 8 == 0.  With gridDim.z > 1 (the weight gradients,
// K = the batch) each CTA takes a slice of K and adds its partial sums to Z (zeroed by the caller).
constexpr int kGtM = 128, kGtN = 128, kGtK = 64;
constexpr size_t kGtStageA = (size_t)kGtM * kGtK * 2, kGtStageB = (size_t)kGtN * kGtK * 2;
constexpr size_t kGtSmem = 2 * (kGtStageA + kGtStageB) + 2 * 8 + 16;

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}

__global__ void __launch_bounds__(kGtM, 1) k_gemm_nt_tc(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B,
                                                       int ldb, int M, int N, int K, const float *__restrict__ bias,
                                                       float *Z, int ldz, bf16 *H, int ldh, int act, int32_t *err) {
  extern __shared__ __align__(1024) unsigned char gt_smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(gt_smem + 2 * (kGtStageA + kGtStageB));
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * kGtM, n0 = blockIdx.x * kGtN;
  const int nt = min(kGtN, ((N - n0 + 15) / 16) * 16);  // this CTA's columns, a multiple of 16
  const uint32_t ncols = nt <= 32 ? 32u : (nt <= 64 ? 64u : 128u);
  if (tid == 0) {
    for (int b = 0; b < 2; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc(nt);
  // this CTA's K slice, whole steps of kGtK
  const int steps = (K + kGtK - 1) / kGtK, per = (steps + gridDim.z - 1) / gridDim.z;
  const int kbeg = blockIdx.z * per * kGtK, kend = min(K, kbeg + per * kGtK);
  const int nk = kend > kbeg ? (kend - kbeg + kGtK - 1) / kGtK : 0;
  uint32_t phase[2] = {0u, 0u};
  bool ok = true;
  int pending = 0;  // stages with an MMA not yet waited for (bit per stage)
  for (int ks = 0; ks < nk && ok; ks++) {
    const int st = ks & 1;
    unsigned char *sa = gt_smem + st * (kGtStageA + kGtStageB), *sb = sa + kGtStageA;
    if (pending & (1 << st)) {  // the MMA that read this stage two steps ago
      ok = mbar_wait(smem_u32(&bars[st]), phase[st]);
      phase[st] ^= 1u;
      pending &= ~(1 << st);
      ok = __syncthreads_and(ok);
      if (!ok) break;
    }
    const int k0 = kbeg + ks * kGtK, kc = min(kGtK, kend - k0);  // kc: a multiple of 16
    // A: 128 rows x kc / 8 chunks; B: nt rows x kc / 8 chunks
    for (int i = tid; i < kGtM * (kc / 8); i += kGtM) {
      const int r = i / (kc / 8), c = i % (kc / 8);
      const uint32_t dst = smem_u32(sa + umma_off(r, 8 * c, kGtM));
      if (m0 + r < M) cp_async16(dst, A + (int64_t)(m0 + r) * lda + k0 + 8 * c);
      else *reinterpret_cast<uint4 *>(sa + umma_off(r, 8 * c, kGtM)) = make_uint4(0u, 0u, 0u, 0u);
    }
    for (int i = tid; i < nt * (kc / 8); i += kGtM) {
      const int r = i / (kc / 8), c = i % (kc / 8);
      const uint32_t dst = smem_u32(sb + umma_off(r, 8 * c, nt));
      if (n0 + r < N) cp_async16(dst, B + (int64_t)(n0 + r) * ldb + k0 + 8 * c);
      else *reinterpret_cast<uint4 *>(sb + umma_off(r, 8 * c, nt)) = make_uint4(0u, 0u, 0u, 0u);
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t lbo_a = (kGtM / 8) * 128, lbo_b = (uint32_t)(nt / 8) * 128;
      const uint32_t a_base = smem_u32(sa), b_base = smem_u32(sb);
      for (int s16 = 0; s16 < kc / 16; s16++) {
        const uint64_t ad = umma_desc(a_base + 2 * s16 * lbo_a, lbo_a, 128);
        const uint64_t bd = umma_desc(b_base + 2 * s16 * lbo_b, lbo_b, 128);
        umma_bf16(tmem, ad, bd, idesc, (ks > 0 || s16 > 0) ? 1u : 0u);
      }
      umma_commit(smem_u32(&bars[st]));
    }
    pending |= 1 << st;
  }
  // the last MMAs
  for (int st = 0; st < 2; st++)
    if (pending & (1 << st)) {
      const bool w = mbar_wait(smem_u32(&bars[st]), phase[st]);
      ok = ok && w;
    }
  ok = __syncthreads_and(ok);
  tc_fence_after();
  if (ok && nk > 0) {
    // epilogue: thread = row m0 + tid (TMEM lane), 16 columns at a time
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    const int r = m0 + tid;
    const bool split = gridDim.z > 1;
    for (int c0 = 0; c0 < nt; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_base + (uint32_t)c0, v);
      if (r < M) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int c = n0 + c0 + j;
          if (c >= N) continue;
          if (split) {
            atomicAdd(Z + (int64_t)r * ldz + c, v[j]);
            continue;
          }
          const float z = v[j] + (bias ? bias[c] : 0.f);
          if (Z) Z[(int64_t)r * ldz + c] = z;
          if (H) H[(int64_t)r * ldh + c] = __float2bfloat16_rn(act ? gelu_f(z) : z);
        }
      }
    }
  } else if (!ok && tid == 0) {
    atomicOr(err, 1 << CUBE_ERR_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
}

// ---------------------------------------------------------------------------------------------
// host side

void launch_mlp_pos(const Lay &L, const int16_t *xp, const int32_t *rhoc, const int64_t *cell_base, float4 *pos,
                    cudaStream_t s) {
  MlpPosK p;
  p.nt = L.nt;
  p.nte = L.nte;
  p.ncb = L.ncb;
  p.nnt = L.nnt;
  p.rcs = L.rcs;
  p.ng = L.ng;
  p.ncells = (int64_t)L.ntile * L.nte * L.nte * L.nte;
  p.xp = xp;
  p.rhoc = rhoc;
  p.cell_base = cell_base;
  p.pos = pos;
  k_mlp_pos<<<(unsigned)((p.ncells + kWarps - 1) / kWarps), kWarps * 32, 0, s>>>(p);
}

// the network reads log(1 + rho): transformed once per cell rather than per stencil read
__global__ void k_mlp_log1p(float *rho, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rho[i] = log1pf(rho[i]);
}

void launch_mlp_density(const float4 *pos, int64_t n, int ng, float *rho, cudaStream_t s) {
  cudaMemsetAsync(rho, 0, sizeof(float) * (size_t)ng * ng * ng, s);
  k_mlp_cic<<<148 * 8, 256, 0, s>>>(pos, n, ng, rho);
  k_mlp_log1p<<<148 * 8, 256, 0, s>>>(rho, (int64_t)ng * ng * ng);
}

void launch_mlp_features(const float4 *pos, int64_t n, const float *rho, int ng, bf16 *X, cudaStream_t s) {
  k_mlp_features<<<148 * 8, 256, 0, s>>>(pos, n, rho, ng, X);
}

// The training GEMMs run on tcgen05 (k_gemm_nt_tc); CUBE_MLP_MMA_SYNC selects the mma.sync
// kernel instead (kept as an independent cross-check).
static int32_t *g_gemm_err = nullptr;  // status word of the current training call (MlpParams::err)

void launch_gemm_nt(const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, const float *bias, float *Z,
                    int ldz, bf16 *H, int ldh, int act, cudaStream_t s) {
  if (!getenv("CUBE_MLP_MMA_SYNC") && g_gemm_err) {
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
      cudaFuncSetAttribute(k_gemm_nt_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGtSmem);
      attr_dev = dev;
    }
    // long K (the weight gradients sum over the batch) on few output tiles: split K over CTAs
    int split = 1;
    if (Z && !H && !bias && !act && M <= 2 * kGtM && K >= 4 * kGtK) split = std::min(32, K / (4 * kGtK));
    if (split > 1) cudaMemset2DAsync(Z, sizeof(float) * (size_t)ldz, 0, sizeof(float) * (size_t)N, (size_t)M, s);
    dim3 grid((unsigned)((N + kGtN - 1) / kGtN), (unsigned)((M + kGtM - 1) / kGtM), (unsigned)split);
    k_gemm_nt_tc<<<grid, kGtM, kGtSmem, s>>>(A, lda, B, ldb, M, N, K, bias, Z, ldz, H, ldh, act, g_gemm_err);
    return;
  }
  dim3 grid((unsigned)((N + kGT - 1) / kGT), (unsigned)((M + kGT - 1) / kGT));
  k_gemm_nt<<<grid, 128, 0, s>>>(A, lda, B, ldb, M, N, K, bias, Z, ldz, H, ldh, act);
}

void launch_mlp_apply(const MlpParams &m, const float4 *pos, const float *rho, int ng, int64_t n, float *vp,
                      float coef, int num_sms, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kApplySmem);
    cudaFuncSetAttribute(k_mlp_apply_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    attr = true;
  }
  MlpApplyK p{m.wb, m.master, pos, rho, ng, n, vp, coef};
  if (getenv("CUBE_MLP_MMA_SYNC")) {
    k_mlp_apply<<<num_sms, kApplyWarps * 32, kApplySmem, s>>>(p);
  } else {
    k_mlp_apply_tc<<<num_sms, kTcThreads, kTcSmem, s>>>(p, m.err);
  }
}

// Forward + backward + Adam on one batch of `batch` rows picked by `rows` from X / T.
int mlp_train_step(MlpParams &m, const bf16 *X, const float *T, const int32_t *rows, int batch, float lr,
                   float *loss, cudaStream_t s) {
  if (batch <= 0 || batch > m.cap || batch % 16) return CUBE_ERR_INVALID;
  g_gemm_err = m.err;
  const int B = batch, W = kMlpW, OP = kMlpOutPad;
  const int g1 = 148 * 8;
  k_mlp_gather<<<g1, 256, 0, s>>>(X, T, rows, B, m.xb, m.tb);
  // forward, keeping the pre-activations and the BF16 layer inputs
  launch_gemm_nt(m.xb, kMlpK1, m.wb + mlp_wboff(0), kMlpK1, B, W, kMlpK1, m.master + mlp_boff(0), m.z[0], W,
                 m.a[0], W, 1, s);
  launch_gemm_nt(m.a[0], W, m.wb + mlp_wboff(1), W, B, W, W, m.master + mlp_boff(1), m.z[1], W, m.a[1], W, 1, s);
  launch_gemm_nt(m.a[1], W, m.wb + mlp_wboff(2), W, B, W, W, m.master + mlp_boff(2), m.z[2], W, m.a[2], W, 1, s);
  cudaMemsetAsync(m.b4pad, 0, sizeof(float) * OP, s);
  cudaMemcpyAsync(m.b4pad, m.master + mlp_boff(3), sizeof(float) * kMlpOut, cudaMemcpyDeviceToDevice, s);
  launch_gemm_nt(m.a[2], W, m.wb + mlp_wboff(3), W, B, OP, W, m.b4pad, m.y, OP, nullptr, 0, 0, s);
  k_mse<<<g1, 256, 0, s>>>(m.y, m.tb, B, m.dy, m.dyb, loss);
  // gradients, written into m.grad in the master layout
  float *gw[4] = {m.grad + mlp_woff(0), m.grad + mlp_woff(1), m.grad + mlp_woff(2), m.grad + mlp_woff(3)};
  float *gb[4] = {m.grad + mlp_boff(0), m.grad + mlp_boff(1), m.grad + mlp_boff(2), m.grad + mlp_boff(3)};
  const dim3 tb(32, 8);
  auto transpose = [&](const bf16 *in, int R, int C, bf16 *out) {
    k_transpose_bf16<<<dim3((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32)), tb, 0, s>>>(in, R, C, out);
  };
  // layer 4: dW4 = dY^T a3 (rows 0..2 kept), db4 = column sums of dY, da3 = dY W4
  transpose(m.dyb, B, OP, m.dzt);
  transpose(m.a[2], B, W, m.at);
  launch_gemm_nt(m.dzt, B, m.at, B, kMlpOut, W, B, nullptr, gw[3], W, nullptr, 0, 0, s);
  k_colsum<<<1, 256, 0, s>>>(m.dy, B, OP, kMlpOut, gb[3]);
  launch_gemm_nt(m.dyb, OP, m.wt + mlp_wboff(3), OP, B, W, OP, nullptr, m.da, W, nullptr, 0, 0, s);
  for (int l = 2; l >= 0; --l) {
    const int K = mlp_K(l);
    k_gelu_bwd<<<g1, 256, 0, s>>>(m.da, m.z[l], (int64_t)B * W, m.dz, m.dzb);
    k_colsum<<<W / 32, 256, 0, s>>>(m.dz, B, W, W, gb[l]);
    transpose(m.dzb, B, W, m.dzt);
    const bf16 *prev = l ? m.a[l - 1] : m.xb;
    transpose(prev, B, K, m.at);
    launch_gemm_nt(m.dzt, B, m.at, B, W, K, B, nullptr, gw[l], K, nullptr, 0, 0, s);
    if (l) launch_gemm_nt(m.dzb, W, m.wt + mlp_wboff(l), W, B, K, W, nullptr, m.da, W, nullptr, 0, 0, s);
  }
  m.step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)m.step), c2 = 1.f - powf(b2, (float)m.step);
  k_adam<<<g1, 256, 0, s>>>(m.master, m.grad, m.mom, m.vel, kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
  k_mlp_pack<<<g1, 256, 0, s>>>(m.master, m.wb, m.wt);
  return cudaGetLastError() == cudaSuccess ? CUBE_OK : CUBE_ERR_CUDA;
}

// Y[rows][3] of X through the training GEMM path (no kick): for checks against the oracle
int mlp_forward(MlpParams &m, const bf16 *X, int64_t nrows, float *Y, cudaStream_t s) {
  g_gemm_err = m.err;
  const int W = kMlpW, OP = kMlpOutPad;
  cudaMemsetAsync(m.b4pad, 0, sizeof(float) * OP, s);
  cudaMemcpyAsync(m.b4pad, m.master + mlp_boff(3), sizeof(float) * kMlpOut, cudaMemcpyDeviceToDevice, s);
  for (int64_t r0 = 0; r0 < nrows; r0 += m.cap) {
    const int B = (int)std::min<int64_t>(m.cap, nrows - r0);
    launch_gemm_nt(X + r0 * kMlpK1, kMlpK1, m.wb + mlp_wboff(0), kMlpK1, B, W, kMlpK1, m.master + mlp_boff(0),
                   nullptr, 0, m.a[0], W, 1, s);
    launch_gemm_nt(m.a[0], W, m.wb + mlp_wboff(1), W, B, W, W, m.master + mlp_boff(1), nullptr, 0, m.a[1], W, 1, s);
    launch_gemm_nt(m.a[1], W, m.wb + mlp_wboff(2), W, B, W, W, m.master + mlp_boff(2), nullptr, 0, m.a[2], W, 1, s);
    launch_gemm_nt(m.a[2], W, m.wb + mlp_wboff(3), W, B, kMlpOut, W, m.b4pad, Y + r0 * kMlpOut, kMlpOut, nullptr, 0,
                   0, s);
  }
  return cudaGetLastError() == cudaSuccess ? CUBE_OK : CUBE_ERR_CUDA;
}

void launch_mlp_pack(MlpParams &m, cudaStream_t s) { k_mlp_pack<<<148 * 8, 256, 0, s>>>(m.master, m.wb, m.wt); }

}  // namespace cube
