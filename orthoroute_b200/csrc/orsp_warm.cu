// Kernels of the learned history warm start: a small 3D convolutional net on
// the routing grid (channels-last bf16 activations [D][H][W][C], C a multiple
// of 16), trained and run with these kernels only.
//
//   conv3d_kernel      3x3x3 convolution as an implicit GEMM on the tensor
//                      cores (bf16 in, fp32 accumulate): M = voxels, N = output
//                      channels, K = 27 taps x input channels.  Fused bias,
//                      ReLU and (for the backward pass) the ReLU mask of the
//                      layer's output applied to the incoming gradient.
//   wgrad_kernel       weight gradient dW[tap][ci][co] = sum_v X[v+tap][ci] G[v][co],
//                      a GEMM with K = voxels, split over blocks, fp32 atomics.
//   small kernels      bias gradient, 2x2 average pooling and nearest
//                      upsampling in x/y (and their adjoints), add, MSE loss,
//                      Adam, bf16 weight packing.
// The backward pass of a convolution with respect to its input is the same
// convolution with the taps mirrored and the channel roles swapped
// (pack_weights with transpose = 1).
#include <mma.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "orsp_warm.h"

using namespace nvcuda;

namespace {

constexpr int CONV_TILE = 64;  // voxels along x per block
constexpr int CONV_THREADS = 128;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// Y[v][co] = act(bias[co] + sum_{tap, ci} Xm[v + tap][ci] W[tap][ci][co]),
// Xm = X, or X * (M > 0) when a mask M (same layout as X) is given.
// Zero padding outside the grid.  Cin % 16 == 0, Cout % 16 == 0, Cout <= 64.
__global__ void __launch_bounds__(CONV_THREADS) conv3d_kernel(
    const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ M, const __nv_bfloat16 *__restrict__ Wt,
    const float *__restrict__ bias, __nv_bfloat16 *__restrict__ Y, float *__restrict__ Yf, int D, int H, int W,
    int Cin, int Cout, int relu) {
  __shared__ __align__(32) __nv_bfloat16 sA[CONV_TILE * 16];
  __shared__ __align__(32) __nv_bfloat16 sB[16 * 64];
  __shared__ __align__(32) float sC[CONV_TILE * 64];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * CONV_TILE, y = blockIdx.y % H, z = blockIdx.y / H;
  const int nt = Cout / 16;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) wmma::fill_fragment(acc[j], 0.0f);
  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const int zz = z + dz, yy = y + dy;
    const bool plane_ok = zz >= 0 && zz < D && yy >= 0 && yy < H;
    for (int c0 = 0; c0 < Cin; c0 += 16) {
      // A: 64 voxels x 16 channels, 16 bytes per thread
      {
        const int row = tid >> 1, half = tid & 1;
        const int xx = x0 + row + dx;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (plane_ok && xx >= 0 && xx < W && x0 + row < W) {
          const int64_t off = (((int64_t)zz * H + yy) * W + xx) * Cin + c0 + half * 8;
          v = *reinterpret_cast<const uint4 *>(X + off);
          if (M) {
            const uint4 m = *reinterpret_cast<const uint4 *>(M + off);
            __nv_bfloat16 *pv = reinterpret_cast<__nv_bfloat16 *>(&v);
            const __nv_bfloat16 *pm = reinterpret_cast<const __nv_bfloat16 *>(&m);
#pragma unroll
            for (int q = 0; q < 8; ++q)
              if (!(bf(pm[q]) > 0.0f)) pv[q] = __float2bfloat16(0.0f);
          }
        }
        *reinterpret_cast<uint4 *>(sA + row * 16 + half * 8) = v;
      }
      // B: 16 input channels x Cout
      for (int i = tid; i < 16 * Cout / 8; i += CONV_THREADS) {
        const int k = (i * 8) / Cout, n = (i * 8) % Cout;
        *reinterpret_cast<uint4 *>(sB + k * Cout + n) =
            *reinterpret_cast<const uint4 *>(Wt + ((int64_t)tap * Cin + c0 + k) * Cout + n);
      }
      __syncthreads();
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
      wmma::load_matrix_sync(fa, sA + warp * 16 * 16, 16);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (j < nt) {
          wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
          wmma::load_matrix_sync(fb, sB + j * 16, Cout);
          wmma::mma_sync(acc[j], fa, fb, acc[j]);
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (j < nt) wmma::store_matrix_sync(sC + warp * 16 * Cout + j * 16, acc[j], Cout, wmma::mem_row_major);
  __syncthreads();
  for (int i = tid; i < CONV_TILE * Cout; i += CONV_THREADS) {
    const int row = i / Cout, co = i % Cout;
    const int xx = x0 + row;
    if (xx >= W) continue;
    float v = sC[i] + (bias ? bias[co] : 0.0f);
    if (relu) v = fmaxf(v, 0.0f);
    const int64_t o = (((int64_t)z * H + y) * W + xx) * Cout + co;
    if (Yf) Yf[o] = v;
    else Y[o] = __float2bfloat16(v);
  }
}

// dW[tap][ci][co] += sum_v X[v + tap][ci] * G[v][co], with G = dY, or
// dY * (Y > 0) when the layer's output Y is given.  Block: one tap, `rows`
// consecutive (z, y) rows; 16 voxels per k-step.  Cin, Cout multiples of 16,
// at most 64 each.
__global__ void __launch_bounds__(CONV_THREADS) wgrad_kernel(
    const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ dY, const __nv_bfloat16 *__restrict__ Yo,
    float *__restrict__ dW, int D, int H, int W, int Cin, int Cout, int rows) {
  __shared__ __align__(32) __nv_bfloat16 sX[16 * 64];
  __shared__ __align__(32) __nv_bfloat16 sG[16 * 64];
  __shared__ __align__(32) float sC[64 * 64];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tap = blockIdx.y;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const int mt = Cin / 16, nt = Cout / 16;
  const int ntile = mt * nt;  // <= 16; warp w owns tiles w, w+4, w+8, w+12
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) wmma::fill_fragment(acc[j], 0.0f);
  const int r0 = blockIdx.x * rows, r1 = min(r0 + rows, D * H);
  for (int r = r0; r < r1; ++r) {
    const int z = r / H, y = r % H;
    const int zz = z + dz, yy = y + dy;
    const bool plane_ok = zz >= 0 && zz < D && yy >= 0 && yy < H;
    for (int xb = 0; xb < W; xb += 16) {
      // X tile: 16 voxels (shifted by the tap) x Cin; G tile: 16 voxels x Cout
      for (int i = tid; i < 16 * Cin / 8; i += CONV_THREADS) {
        const int v = (i * 8) / Cin, c = (i * 8) % Cin;
        const int x = xb + v, xx = x + dx;
        uint4 q = make_uint4(0, 0, 0, 0);
        if (plane_ok && x < W && xx >= 0 && xx < W)
          q = *reinterpret_cast<const uint4 *>(X + (((int64_t)zz * H + yy) * W + xx) * Cin + c);
        *reinterpret_cast<uint4 *>(sX + v * Cin + c) = q;
      }
      for (int i = tid; i < 16 * Cout / 8; i += CONV_THREADS) {
        const int v = (i * 8) / Cout, c = (i * 8) % Cout;
        const int x = xb + v;
        uint4 q = make_uint4(0, 0, 0, 0);
        if (x < W) {
          const int64_t off = (((int64_t)z * H + y) * W + x) * Cout + c;
          q = *reinterpret_cast<const uint4 *>(dY + off);
          if (Yo) {
            const uint4 m = *reinterpret_cast<const uint4 *>(Yo + off);
            __nv_bfloat16 *pq = reinterpret_cast<__nv_bfloat16 *>(&q);
            const __nv_bfloat16 *pm = reinterpret_cast<const __nv_bfloat16 *>(&m);
#pragma unroll
            for (int t = 0; t < 8; ++t)
              if (!(bf(pm[t]) > 0.0f)) pq[t] = __float2bfloat16(0.0f);
          }
        }
        *reinterpret_cast<uint4 *>(sG + v * Cout + c) = q;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int t = warp + 4 * j;
        if (t < ntile) {
          const int mi = t / nt, ni = t % nt;
          // A = X^T (Cin x 16 voxels): X tile is voxel-major, i.e. A column-major
          wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> fa;
          wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
          wmma::load_matrix_sync(fa, sX + mi * 16, Cin);
          wmma::load_matrix_sync(fb, sG + ni * 16, Cout);
          wmma::mma_sync(acc[j], fa, fb, acc[j]);
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int t = warp + 4 * j;
    if (t < ntile) {
      const int mi = t / nt, ni = t % nt;
      wmma::store_matrix_sync(sC + (mi * 16) * Cout + ni * 16, acc[j], Cout, wmma::mem_row_major);
    }
  }
  __syncthreads();
  for (int i = tid; i < Cin * Cout; i += CONV_THREADS) atomicAdd(&dW[(int64_t)tap * Cin * Cout + i], sC[i]);
}

// db[co] += sum_v G[v][co] (G as in wgrad_kernel).
__global__ void bias_grad_kernel(const __nv_bfloat16 *__restrict__ dY, const __nv_bfloat16 *__restrict__ Yo,
                                 float *__restrict__ db, int64_t nvox, int C) {
  __shared__ float s[64 * 4];
  const int c = threadIdx.x % C, lane_group = threadIdx.x / C, groups = blockDim.x / C;
  float acc = 0.0f;
  for (int64_t v = (int64_t)blockIdx.x * groups + lane_group; v < nvox; v += (int64_t)gridDim.x * groups) {
    const float g = bf(dY[v * C + c]);
    if (!Yo || bf(Yo[v * C + c]) > 0.0f) acc += g;
  }
  if (lane_group < 4 && threadIdx.x < groups * C) s[lane_group * C + c] = 0.0f;
  __syncthreads();
  atomicAdd(&s[(lane_group % 4) * C + c], acc);
  __syncthreads();
  if (threadIdx.x < C) atomicAdd(&db[c], s[c] + s[C + c] + s[2 * C + c] + s[3 * C + c]);
}

// 2x2 average over x, y (H, W even): out [D][H/2][W/2][C].
__global__ void pool_kernel(const __nv_bfloat16 *__restrict__ X, __nv_bfloat16 *__restrict__ Y, int D, int H, int W,
                            int C) {
  const int64_t n = (int64_t)D * (H / 2) * (W / 2) * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int64_t r = i / C;
    const int x = (int)(r % (W / 2));
    r /= (W / 2);
    const int y = (int)(r % (H / 2));
    const int z = (int)(r / (H / 2));
    const int64_t b = (((int64_t)z * H + 2 * y) * W + 2 * x) * C + c;
    const float s = bf(X[b]) + bf(X[b + C]) + bf(X[b + (int64_t)W * C]) + bf(X[b + (int64_t)W * C + C]);
    Y[i] = __float2bfloat16(0.25f * s);
  }
}

// Adjoint of pool_kernel: dX[fine] = dY[coarse] / 4.  Also nearest upsampling
// (scale 1): out[fine] = in[coarse].  Fine grid [D][H][W][C].
__global__ void spread_kernel(const __nv_bfloat16 *__restrict__ Yc, __nv_bfloat16 *__restrict__ Xf, int D, int H,
                              int W, int C, float scale) {
  const int64_t n = (int64_t)D * H * W * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int64_t r = i / C;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int z = (int)(r / H);
    Xf[i] = __float2bfloat16(scale * bf(Yc[(((int64_t)z * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]));
  }
}

// Adjoint of nearest upsampling: dCoarse = sum of the 4 fine gradients.
__global__ void gather4_kernel(const __nv_bfloat16 *__restrict__ Xf, __nv_bfloat16 *__restrict__ Yc, int D, int H,
                               int W, int C) {
  const int64_t n = (int64_t)D * (H / 2) * (W / 2) * C;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int64_t r = i / C;
    const int x = (int)(r % (W / 2));
    r /= (W / 2);
    const int y = (int)(r % (H / 2));
    const int z = (int)(r / (H / 2));
    const int64_t b = (((int64_t)z * H + 2 * y) * W + 2 * x) * C + c;
    Yc[i] = __float2bfloat16(bf(Xf[b]) + bf(Xf[b + C]) + bf(Xf[b + (int64_t)W * C]) + bf(Xf[b + (int64_t)W * C + C]));
  }
}

__global__ void add_kernel(const __nv_bfloat16 *a, const __nv_bfloat16 *b, __nv_bfloat16 *out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(bf(a[i]) + bf(b[i]));
}

// Mean squared error over the first `used` of C channels of an fp32 output,
// with a per-voxel weight (nullptr = 1).  loss[0] += sum w (p - t)^2 / count;
// dP (bf16, C channels) = 2 w (p - t) / count on used channels, 0 elsewhere.
__global__ void mse_kernel(const float *__restrict__ P, const float *__restrict__ T, const float *__restrict__ wv,
                           __nv_bfloat16 *__restrict__ dP, float *__restrict__ loss, int64_t nvox, int C, int used,
                           float inv_count) {
  float acc = 0.0f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox * C; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t v = i / C;
    float g = 0.0f;
    if (c < used) {
      const float d = P[i] - T[v * used + c];
      const float w = wv ? wv[v] : 1.0f;
      acc += w * d * d;
      g = 2.0f * w * d * inv_count;
    }
    dP[i] = __float2bfloat16(g);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc * inv_count);
}

// Adam on fp32 master weights (bias-corrected step sizes given by the host).
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int64_t n, float lr_t, float b1, float b2, float eps, float wd) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr_t * mi / (sqrtf(vi) + eps);
  }
}

// bf16 weights for conv3d_kernel from fp32 master weights [27][Cin][Cout]:
// transpose = 0: Wt[tap][ci][co] = w[tap][ci][co];
// transpose = 1 (input gradient): Wt[tap][co][ci] = w[26 - tap][ci][co].
__global__ void pack_weights_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ Wt, int Cin, int Cout,
                                    int transpose) {
  const int n = 27 * Cin * Cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int tap = i / (Cin * Cout), r = i % (Cin * Cout), ci = r / Cout, co = r % Cout;
    if (!transpose) Wt[i] = __float2bfloat16(w[i]);
    else Wt[((int64_t)(26 - tap) * Cout + co) * Cin + ci] = __float2bfloat16(w[i]);
  }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

using namespace orsp;

extern "C" int orsp_warm_conv3d(const void *X, const void *mask, const void *Wt, const float *bias, void *Y,
                                float *Yf, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout, int32_t relu,
                                uintptr_t stream) {
  if (!X || !Wt || (!Y && !Yf) || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cin % 16 || Cout <= 0 || Cout % 16 ||
      Cout > 64) {
    set_error("warm_conv3d: bad arguments (Cin, Cout multiples of 16, Cout <= 64)");
    return ORSP_ERR_ARG;
  }
  dim3 grid((W + CONV_TILE - 1) / CONV_TILE, (unsigned)(D * H));
  conv3d_kernel<<<grid, CONV_THREADS, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)X, (const __nv_bfloat16 *)mask, (const __nv_bfloat16 *)Wt, bias, (__nv_bfloat16 *)Y, Yf,
      D, H, W, Cin, Cout, relu);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_wgrad(const void *X, const void *dY, const void *Yo, float *dW, float *db, int32_t D,
                               int32_t H, int32_t W, int32_t Cin, int32_t Cout, uintptr_t stream) {
  if (!X || !dY || !dW || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cin % 16 || Cin > 64 || Cout <= 0 ||
      Cout % 16 || Cout > 64) {
    set_error("warm_wgrad: bad arguments (Cin, Cout multiples of 16, at most 64)");
    return ORSP_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int rows_total = D * H;
  const int rows = std::max(1, rows_total / 256);
  dim3 grid((rows_total + rows - 1) / rows, 27);
  wgrad_kernel<<<grid, CONV_THREADS, 0, st>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)dY,
                                              (const __nv_bfloat16 *)Yo, dW, D, H, W, Cin, Cout, rows);
  ORSP_CUDA(cudaGetLastError());
  if (db) {
    const int64_t nvox = (int64_t)D * H * W;
    const int threads = (256 / Cout) * Cout;
    bias_grad_kernel<<<grid_for(nvox * Cout), threads, 0, st>>>((const __nv_bfloat16 *)dY, (const __nv_bfloat16 *)Yo,
                                                                db, nvox, Cout);
    ORSP_CUDA(cudaGetLastError());
  }
  return ORSP_OK;
}

extern "C" int orsp_warm_pool(const void *X, void *Y, int32_t D, int32_t H, int32_t W, int32_t C, uintptr_t stream) {
  if (!X || !Y || H % 2 || W % 2 || C <= 0) { set_error("warm_pool: even H, W required"); return ORSP_ERR_ARG; }
  const int64_t n = (int64_t)D * (H / 2) * (W / 2) * C;
  pool_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)X, (__nv_bfloat16 *)Y, D, H, W,
                                                             C);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_spread(const void *Yc, void *Xf, int32_t D, int32_t H, int32_t W, int32_t C, float scale,
                                uintptr_t stream) {
  if (!Yc || !Xf || H % 2 || W % 2 || C <= 0) { set_error("warm_spread: even H, W required"); return ORSP_ERR_ARG; }
  const int64_t n = (int64_t)D * H * W * C;
  spread_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)Yc, (__nv_bfloat16 *)Xf, D, H,
                                                               W, C, scale);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_gather4(const void *Xf, void *Yc, int32_t D, int32_t H, int32_t W, int32_t C,
                                 uintptr_t stream) {
  if (!Xf || !Yc || H % 2 || W % 2 || C <= 0) { set_error("warm_gather4: even H, W required"); return ORSP_ERR_ARG; }
  const int64_t n = (int64_t)D * (H / 2) * (W / 2) * C;
  gather4_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)Xf, (__nv_bfloat16 *)Yc, D, H,
                                                                W, C);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_add(const void *a, const void *b, void *out, int64_t n, uintptr_t stream) {
  if (!a || !b || !out || n < 0) { set_error("warm_add: bad arguments"); return ORSP_ERR_ARG; }
  add_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)a, (const __nv_bfloat16 *)b,
                                                            (__nv_bfloat16 *)out, n);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_mse(const float *P, const float *T, const float *wv, void *dP, float *loss, int64_t nvox,
                             int32_t C, int32_t used, float inv_count, uintptr_t stream) {
  if (!P || !T || !dP || !loss || used <= 0 || used > C) { set_error("warm_mse: bad arguments"); return ORSP_ERR_ARG; }
  mse_kernel<<<grid_for(nvox * C), 256, 0, (cudaStream_t)stream>>>(P, T, wv, (__nv_bfloat16 *)dP, loss, nvox, C, used,
                                                                    inv_count);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr_t, float b1, float b2,
                              float eps, float wd, uintptr_t stream) {
  if (!w || !g || !m || !v || n < 0) { set_error("warm_adam: bad arguments"); return ORSP_ERR_ARG; }
  adam_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr_t, b1, b2, eps, wd);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_pack_weights(const float *w, void *Wt, int32_t Cin, int32_t Cout, int32_t transpose,
                                      uintptr_t stream) {
  if (!w || !Wt || Cin <= 0 || Cout <= 0) { set_error("warm_pack_weights: bad arguments"); return ORSP_ERR_ARG; }
  pack_weights_kernel<<<grid_for(27 * Cin * Cout), 256, 0, (cudaStream_t)stream>>>(w, (__nv_bfloat16 *)Wt, Cin, Cout,
                                                                                   transpose);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}
