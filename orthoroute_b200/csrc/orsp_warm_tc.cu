// The warm-start network's 3x3x3 convolution on the 5th-generation tensor
// cores: tcgen05.mma (kind::f16, bf16 operands, fp32 accumulator in TMEM).
//
// Implicit GEMM, as conv3d_kernel in orsp_warm.cu: M = 128 voxels along x of
// one (z, y) row, N = Cout, K = 27 taps x Cin.  Each CTA is persistent:
//   - it stages every tap's weights once, B[n][k] = Wt[tap][k][n], in shared
//     memory in the K-major canonical UMMA layout without swizzle (core
//     matrices of 8 rows x 16 bytes, rows contiguous; the two 8-element halves
//     of a 16-wide K slice 128 bytes apart, 8-row groups 256 bytes apart);
//   - per tile, nine stages (dz, dy): 256 threads copy one input row once
//     into a stage buffer (cp.async, zero outside the grid; the optional ReLU
//     mask through registers), whose 16-byte rows serve the three (dx) taps
//     A[m][k] = X[z+dz][y+dy][x0+m+dx][k] as descriptors one row apart, and
//     one thread issues the 3 x Cin/16 MMAs (K = 16 each) into the TMEM
//     accumulator and commits them to the buffer's mbarrier, while the copies
//     of the next stages are in flight (a ring of up to six buffers);
//   - the epilogue reads the accumulator with tcgen05.ld (warps w and w + 4
//     share TMEM lanes 32 (w % 4) .., i.e. those voxels, and split the output
//     channels), adds the bias, applies the ReLU and stores bf16 or fp32.
// The weight gradient (wgrad_tc_kernel) is a second tcgen05 GEMM.
// Every mbarrier wait is bounded by the global timer; on expiry the kernel
// records an error, waits once more (bounded) for its MMAs, frees its TMEM
// and returns.  Single-GPU code: no TMA, no multicast.
#include <cstdlib>
#include <algorithm>
#include <climits>
#include <cstdint>

#include <cuda_bf16.h>

#include "common.cuh"
#include "orsp_warm.h"

namespace {

constexpr int TC_M = 128;        // voxels per tile: the MMA's M and the accumulator's TMEM lanes
constexpr int TC_THREADS = 128;  // four warps, one per 32-lane quarter of TMEM
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

__device__ int g_tc_err = 0;     // set by a kernel whose wait expired (orsp_warm_tc_status)

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major operand without swizzle:
// start address, leading byte offset (between the K halves), stride byte
// offset (between 8-row groups), all in 16-byte units; version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor: fp32 accumulator, bf16 A and B, both K-major,
// N >> 3 and M >> 4.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
      "}"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete, at most TC_WAIT_NS.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = dev_globaltimer();
  for (;;) {
    if (mbar_try(bar, parity)) return true;
    if (dev_globaltimer() - t0 > TC_WAIT_NS) return false;
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared memory of the convolution: all weights (27 taps x Cin/16 K slices
// x Cout rows of 32 bytes), NS stage buffers, NS mbarriers and the TMEM
// address slot.  A stage buffer holds one input row of TC_M + 2 voxels as
// Cin / 8 planes (8 channels each) of 16-byte rows, CV_PLANE bytes apart:
// row r of plane cg at cg * CV_PLANE + r * 16.
constexpr int CV_PLANE = (TC_M + 2) * 16;
__host__ __device__ constexpr size_t cv_weight_bytes(int Cin, int Cout) {
  return static_cast<size_t>(27) * (Cin / 16) * Cout * 32;
}
__host__ __device__ constexpr size_t cv_stage_bytes(int Cin) {
  return (static_cast<size_t>(Cin / 8) * CV_PLANE + 127) & ~static_cast<size_t>(127);
}
__host__ __device__ constexpr size_t cv_smem_bytes(int Cin, int Cout, int ns) {
  return cv_weight_bytes(Cin, Cout) + ns * cv_stage_bytes(Cin) + 8 * ns + 64;
}
// Stage buffers that fit beside the weights in 200 KB (at most 6; 0 when
// fewer than 3 fit).
inline int cv_stages(int Cin, int Cout) {
  const size_t budget = 200 * 1024;
  if (cv_smem_bytes(Cin, Cout, 3) > budget) return 0;
  int ns = 3;
  while (ns < 6 && cv_smem_bytes(Cin, Cout, ns + 1) <= budget) ++ns;
  return ns;
}

// 16-byte global -> shared copy that fills zeros when `bytes` is 0.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most n (0..4) of this thread's copy groups are pending.
__device__ __forceinline__ void cp_async_wait(int n) {
  if (n <= 0) asm volatile("cp.async.wait_group 0;" ::: "memory");
  else if (n == 1) asm volatile("cp.async.wait_group 1;" ::: "memory");
  else if (n == 2) asm volatile("cp.async.wait_group 2;" ::: "memory");
  else if (n == 3) asm volatile("cp.async.wait_group 3;" ::: "memory");
  else asm volatile("cp.async.wait_group 4;" ::: "memory");
}

constexpr int CV_THREADS = 256;  // eight warps gather; warps w and w + 4 share TMEM lanes 32 (w % 4)..

// Pipelined implicit GEMM.  A stage is one input row (plane z + dz, row
// y + dy) of a tile: the 130 voxels x0 - 1 .. x0 + 128 are copied once, 16
// bytes at a time with cp.async (zero fill outside the grid), into the
// stage's channel planes.  The A operand of tap dx is that buffer itself: in
// the K-major layout without swizzle, a stride of 128 bytes between 8-row
// core-matrix groups puts row m at 16 m bytes, so the descriptor of tap dx
// starts (dx + 1) rows in (row m of tap dx = voxel x0 + m + dx), with the
// planes of a 16-channel K slice CV_PLANE bytes apart.  One copy serves the
// three taps.  Stages run through a ring of NS buffers: while
// the tensor core consumes stages s - 1 and s, the copies of stages
// s + 1 .. s + NS - 2 are in flight.  Buffer b's mbarrier completes when the MMAs of the stage
// last held in b are done (tcgen05.commit), which is what a refill of b waits
// for; the 9th stage of a tile also releases the epilogue.  With the ReLU
// mask the gather goes through registers (plain loads and shared stores).
// CG = Cin / 8 (2, 4 or 8), a template parameter so that the gather's unit
// arithmetic is resolved at compile time.
template <int CG>
__global__ void __launch_bounds__(CV_THREADS, 1) conv3d_tc_kernel(
    const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ Mk, const __nv_bfloat16 *__restrict__ Wt,
    const float *__restrict__ bias, __nv_bfloat16 *__restrict__ Y, float *__restrict__ Yf, int D, int H, int W,
    int Cin, int Cout, int relu, int NS) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int KC = Cin >> 4;
  const int bblk = Cout * 32;  // bytes of one (tap, 16-wide K slice) weight block
  const size_t SBY = cv_stage_bytes(Cin);
  unsigned char *sB = sm;
  unsigned char *sA = sm + cv_weight_bytes(Cin, Cout);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(sA + NS * SBY);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + NS);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = Cout <= 32 ? 32u : 64u;

  // weights: one 16-byte unit = 8 consecutive k of one n
  const int units_per_tap = Cin * Cout / 8;
  for (int i = tid; i < 27 * units_per_tap; i += CV_THREADS) {
    const int tap = i / units_per_tap, r = i - tap * units_per_tap;
    const int kg = r / Cout, n = r - kg * Cout;  // kg: 8-element group of k
    const __nv_bfloat16 *src = Wt + (static_cast<int64_t>(tap) * Cin + kg * 8) * Cout + n;
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t lo = __bfloat16_as_ushort(src[(2 * j) * Cout]);
      const uint32_t hi = __bfloat16_as_ushort(src[(2 * j + 1) * Cout]);
      v[j] = lo | (hi << 16);
    }
    unsigned char *dst = sB + (tap * KC + (kg >> 1)) * bblk + (n >> 3) * 256 + (kg & 1) * 128 + (n & 7) * 16;
    *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
  }
  if (tid == 0) {
    for (int b = 0; b < NS; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + b)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(TC_M, Cout);

  const int ntx = (W + TC_M - 1) / TC_M;
  const int64_t ntiles = static_cast<int64_t>(D) * H * ntx;
  const int64_t my_tiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int64_t nst = my_tiles * 9;

  // copies of stage s into buffer s % NS (nothing past the last stage); one
  // commit group per call on every thread, so the group counts stay uniform
  // This thread's share of a stage is the same for every stage: units
  // u = tid + j * CV_THREADS of (130 voxels) x CG channel groups, channel
  // group fastest, so a warp reads 512 contiguous bytes and the 8 lanes of a
  // 16-byte store phase hit all 32 banks (planes CV_PLANE = 8 banks apart).
  // Per unit: x offset from x0, element offset in the row, destination.
  constexpr int CIN = CG * 8;
  constexpr int UNITS = (TC_M + 2) * CG;
  constexpr int UPT = (UNITS + CV_THREADS - 1) / CV_THREADS;
  int u_x[UPT], u_off[UPT], u_dst[UPT];
#pragma unroll
  for (int j = 0; j < UPT; ++j) {
    const int i = tid + j * CV_THREADS;
    const int vx = i / CG, cg = i % CG;
    const bool unit = i < UNITS;
    u_x[j] = unit ? vx - 1 : INT_MIN / 2;
    u_off[j] = (vx - 1) * CIN + cg * 8;
    u_dst[j] = unit ? cg * CV_PLANE + vx * 16 : -1;
  }

  // Stage cursors advance by one stage at a time (no division per stage):
  // stage index within the tile (dz * 3 + dy), ring buffer and its phase
  // parity, and the tile with its coordinates (divisions once per tile).
  const int ntiles32 = static_cast<int>(ntiles);
  const int nst32 = static_cast<int>(nst);
  struct Cursor {
    int st9, buf, par, t, tx, y, z;
  };
  auto tile_coords = [&](Cursor &c) {
    c.tx = c.t % ntx;
    const int zy = c.t / ntx;
    c.y = zy % H;
    c.z = zy / H;
  };
  auto advance = [&](Cursor &c) {
    if (++c.buf == NS) {
      c.buf = 0;
      c.par ^= 1;
    }
    if (++c.st9 == 9) {
      c.st9 = 0;
      c.t += gridDim.x;
      if (c.t < ntiles32) tile_coords(c);
    }
  };

  // copies of the stage at cursor ci (nothing past the last stage); one
  // commit group per call on every thread, so the group counts stay uniform
  Cursor ci{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};
  tile_coords(ci);
  int si = 0;  // the stage ci points at
  auto issue = [&]() {
    if (si < nst32) {
      const int zz = ci.z + ci.st9 / 3 - 1, yy = ci.y + ci.st9 % 3 - 1, x0 = ci.tx * TC_M;
      const bool rowok = zz >= 0 && zz < D && yy >= 0 && yy < H;
      unsigned char *buf = sA + static_cast<size_t>(ci.buf) * SBY;
      const __nv_bfloat16 *row = X + ((static_cast<int64_t>(rowok ? zz : 0) * H + (rowok ? yy : 0)) * W + x0) * CIN;
#pragma unroll
      for (int j = 0; j < UPT; ++j) {
        const int xx = x0 + u_x[j];
        const bool in = rowok && xx >= 0 && xx < W;
        const __nv_bfloat16 *src = in ? row + u_off[j] : X;
        if (u_dst[j] < 0) continue;
        if (!Mk) {
          cp_async16(buf + u_dst[j], src, in ? 16 : 0);
        } else {
          uint4 v = make_uint4(0, 0, 0, 0);
          if (in) {
            v = *reinterpret_cast<const uint4 *>(src);
            const uint4 mk = *reinterpret_cast<const uint4 *>(Mk + (src - X));
            __nv_bfloat16 *pv = reinterpret_cast<__nv_bfloat16 *>(&v);
            const __nv_bfloat16 *pm = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
            for (int q = 0; q < 8; ++q)
              if (!(__bfloat162float(pm[q]) > 0.0f)) pv[q] = __float2bfloat16(0.0f);
          }
          *reinterpret_cast<uint4 *>(buf + u_dst[j]) = v;
        }
      }
      advance(ci);
    }
    ++si;
    cp_async_commit();
  };

  // the copies run NS - 2 stages ahead; a buffer is refilled two stages
  // after its MMAs were issued, so their completion is not waited for at once
  for (int k = 0; k < NS - 2; ++k) issue();
  bool ok = true;
  Cursor cc{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};  // the stage consumed
  tile_coords(cc);
  Cursor cw{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};  // two stages behind: the buffer refilled next
  int s = 0, issued_buf = -1, issued_par = 0;  // the last stage whose MMAs were committed
  for (; s < nst32; ++s) {
    const int b = cc.buf;
    const int st9 = cc.st9;
    // this thread's copies of stage s have landed; hand them to the async
    // proxy, then every thread's (and a failed wait anywhere ends the loop)
    cp_async_wait(NS - 3);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    ok = __syncthreads_and(ok ? 1 : 0) != 0;
    tc_fence_after();
    if (!ok) break;
    if (tid == 0) {
      const int tapz = (st9 / 3) * 9 + (st9 % 3) * 3;  // (dz, dy) part of the tap index
#pragma unroll 1
      for (int dxi = 0; dxi < 3; ++dxi)
        for (int kc = 0; kc < KC; ++kc) {
          const uint64_t a =
              umma_smem_desc(smem_addr(sA + b * SBY + (2 * kc) * CV_PLANE + dxi * 16), CV_PLANE, 128);
          const uint64_t bd = umma_smem_desc(smem_addr(sB + ((tapz + dxi) * KC + kc) * bblk), 128, 256);
          mma_bf16(tmem, a, bd, idesc, (st9 | dxi | kc) != 0 ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(bars + b))
                   : "memory");
    }
    issued_buf = b;
    issued_par = cc.par;
    // refill the buffer of stage s - 2 with stage s + NS - 2 once its MMAs
    // are done (for s < 2 that buffer has not been used yet)
    if (s >= 2) {
      ok = mbar_wait(smem_addr(bars + cw.buf), static_cast<uint32_t>(cw.par));
      advance(cw);
    }
    issue();
    if (st9 == 8) {
      // last stage of the tile: the accumulator is final once its MMAs are
      ok = __syncthreads_and((ok && mbar_wait(smem_addr(bars + b), static_cast<uint32_t>(cc.par))) ? 1 : 0) != 0;
      if (!ok) break;
      tc_fence_after();
      const int tx = cc.tx, y = cc.y, z = cc.z;
      // warp w: voxels 32 (w % 4) .. + 31 (its TMEM lanes), channel blocks
      // of 16 starting at 16 (w / 4), every second one
      const int m = (warp & 3) * 32 + lane, xx = tx * TC_M + m;
      for (int c0 = (warp >> 2) * 16; c0 < Cout; c0 += 32) {
        uint32_t r[16];
        tmem_ld16(tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16) + static_cast<uint32_t>(c0), r);
        if (xx < W) {
          const int64_t o = ((static_cast<int64_t>(z) * H + y) * W + xx) * Cout + c0;
          float f[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const float v = __uint_as_float(r[j]) + (bias ? bias[c0 + j] : 0.0f);
            f[j] = relu ? fmaxf(v, 0.0f) : v;
          }
          if (Yf) {
#pragma unroll
            for (int j = 0; j < 16; j += 4)
              *reinterpret_cast<float4 *>(Yf + o + j) = make_float4(f[j], f[j + 1], f[j + 2], f[j + 3]);
          } else {
            uint32_t p[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
              p[j] = static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16(f[2 * j]))) |
                     (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16(f[2 * j + 1]))) << 16);
            *reinterpret_cast<uint4 *>(Y + o) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4 *>(Y + o + 8) = make_uint4(p[4], p[5], p[6], p[7]);
          }
        }
      }
      // the next tile's first MMA overwrites the accumulator: these loads
      // are ordered before it by the next iteration's barrier
      tc_fence_before();
    }
    advance(cc);
  }
  cp_async_wait(0);
  if (!ok) {
    // a wait expired: record it and give the MMAs in flight one more
    // bounded wait (the last stage committed, which completes after all
    // earlier ones) before the accumulator is freed
    if (tid == 0) atomicExch(&g_tc_err, 1);
    if (issued_buf >= 0) mbar_wait(smem_addr(bars + issued_buf), static_cast<uint32_t>(issued_par));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// Warp-specialised form of the same convolution (the default;
// ORSP_WARM_TC_WS=0 selects the kernel above).
// Eight producer warps copy the stages and drain the accumulators; one MMA
// warp (lane 0) issues the tensor-core MMAs.  No block barrier separates the
// stages; per-buffer mbarriers hand them over:
//   full[b]   the producers' copies of the stage in b have landed (256
//             arrivals, each after its thread's cp.async group completed and
//             a proxy fence);
//   empty[b]  the MMAs that read b are done (tcgen05.commit);
//   accf[a]   accumulator a holds a finished tile (tcgen05.commit after the
//             tile's last stage);
//   acce[a]   the producers have read accumulator a (256 arrivals).
// Tiles alternate between two TMEM accumulators, so a tile's epilogue runs
// while the MMAs of the next tile proceed.  The producers signal stage s
// after issuing stage s + LAG (LAG = NS - 2, at most 4); a buffer is refilled
// only after its previous stage's MMAs are done, so the copies of LAG stages
// are in flight while the tensor core consumes.  Every wait is bounded; a
// wait that expires sets a shared abort flag that ends every other wait.
constexpr int WS_PROD = 256;
constexpr int WS_THREADS = WS_PROD + 32;

__host__ __device__ constexpr size_t ws_smem_bytes(int Cin, int Cout, int ns) {
  return cv_weight_bytes(Cin, Cout) + ns * cv_stage_bytes(Cin) + 16 * ns + 64;
}

template <int CG>
__global__ void __launch_bounds__(WS_THREADS, 1) conv3d_tc_ws_kernel(
    const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ Mk, const __nv_bfloat16 *__restrict__ Wt,
    const float *__restrict__ bias, __nv_bfloat16 *__restrict__ Y, float *__restrict__ Yf, int D, int H, int W,
    int Cin, int Cout, int relu, int NS) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ volatile int s_abort;
  const int KC = Cin >> 4;
  const int bblk = Cout * 32;
  const size_t SBY = cv_stage_bytes(Cin);
  unsigned char *sB = sm;
  unsigned char *sA = sm + cv_weight_bytes(Cin, Cout);
  unsigned long long *full = reinterpret_cast<unsigned long long *>(sA + NS * SBY);
  unsigned long long *empty = full + NS;
  unsigned long long *accf = empty + NS;
  unsigned long long *acce = accf + 2;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(acce + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols1 = Cout <= 32 ? 32u : 64u, ncols = 2 * ncols1;

  const int units_per_tap = Cin * Cout / 8;
  for (int i = tid; i < 27 * units_per_tap; i += WS_THREADS) {
    const int tap = i / units_per_tap, r = i - tap * units_per_tap;
    const int kg = r / Cout, n = r - kg * Cout;
    const __nv_bfloat16 *src = Wt + (static_cast<int64_t>(tap) * Cin + kg * 8) * Cout + n;
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t lo = __bfloat16_as_ushort(src[(2 * j) * Cout]);
      const uint32_t hi = __bfloat16_as_ushort(src[(2 * j + 1) * Cout]);
      v[j] = lo | (hi << 16);
    }
    unsigned char *dst = sB + (tap * KC + (kg >> 1)) * bblk + (n >> 3) * 256 + (kg & 1) * 128 + (n & 7) * 16;
    *reinterpret_cast<uint4 *>(dst) = make_uint4(v[0], v[1], v[2], v[3]);
  }
  if (tid == 0) {
    s_abort = 0;
    for (int b = 0; b < NS; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(full + b)), "r"(WS_PROD) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(empty + b)) : "memory");
    }
    for (int a = 0; a < 2; ++a) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(accf + a)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(acce + a)), "r"(WS_PROD) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(TC_M, Cout);

  const int ntx = (W + TC_M - 1) / TC_M;
  const int64_t ntiles = static_cast<int64_t>(D) * H * ntx;
  const int64_t my_tiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int ntiles32 = static_cast<int>(ntiles);
  const int nst32 = static_cast<int>(my_tiles * 9);
  const int my32 = static_cast<int>(my_tiles);
  struct Cursor {
    int st9, buf, par, t, tx, y, z;
  };
  auto tile_coords = [&](Cursor &c) {
    c.tx = c.t % ntx;
    const int zy = c.t / ntx;
    c.y = zy % H;
    c.z = zy / H;
  };
  auto advance = [&](Cursor &c) {
    if (++c.buf == NS) {
      c.buf = 0;
      c.par ^= 1;
    }
    if (++c.st9 == 9) {
      c.st9 = 0;
      c.t += gridDim.x;
      if (c.t < ntiles32) tile_coords(c);
    }
  };
  // a bounded wait that also ends when another role has given up
  auto wait = [&](unsigned long long *bar, int parity) -> bool {
    const uint32_t a = smem_addr(bar);
    const unsigned long long t0 = dev_globaltimer();
    for (;;) {
      if (mbar_try(a, static_cast<uint32_t>(parity))) return true;
      if (s_abort) return false;
      if (dev_globaltimer() - t0 > TC_WAIT_NS) {
        s_abort = 1;
        atomicExch(&g_tc_err, 1);
        return false;
      }
    }
  };
  const int LAG = NS - 2 < 4 ? NS - 2 : 4;

  if (warp < 8) {
    // ------------------------------------------------------------ producers
    constexpr int CIN = CG * 8;
    constexpr int UNITS = (TC_M + 2) * CG;
    constexpr int UPT = (UNITS + WS_PROD - 1) / WS_PROD;
    int u_x[UPT], u_off[UPT], u_dst[UPT];
#pragma unroll
    for (int j = 0; j < UPT; ++j) {
      const int i = tid + j * WS_PROD;
      const int vx = i / CG, cg = i % CG;
      const bool unit = i < UNITS;
      u_x[j] = unit ? vx - 1 : INT_MIN / 2;
      u_off[j] = (vx - 1) * CIN + cg * 8;
      u_dst[j] = unit ? cg * CV_PLANE + vx * 16 : -1;
    }
    auto epilogue = [&](int tx, int y, int z, int acc) {
      const int m = (warp & 3) * 32 + lane, xx = tx * TC_M + m;
      for (int c0 = (warp >> 2) * 16; c0 < Cout; c0 += 32) {
        uint32_t r[16];
        tmem_ld16(tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16) + static_cast<uint32_t>(acc) * ncols1 +
                      static_cast<uint32_t>(c0),
                  r);
        if (xx < W) {
          const int64_t o = ((static_cast<int64_t>(z) * H + y) * W + xx) * Cout + c0;
          float f[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const float v = __uint_as_float(r[j]) + (bias ? bias[c0 + j] : 0.0f);
            f[j] = relu ? fmaxf(v, 0.0f) : v;
          }
          if (Yf) {
#pragma unroll
            for (int j = 0; j < 16; j += 4)
              *reinterpret_cast<float4 *>(Yf + o + j) = make_float4(f[j], f[j + 1], f[j + 2], f[j + 3]);
          } else {
            uint32_t p[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
              p[j] = static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16(f[2 * j]))) |
                     (static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16(f[2 * j + 1]))) << 16);
            *reinterpret_cast<uint4 *>(Y + o) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4 *>(Y + o + 8) = make_uint4(p[4], p[5], p[6], p[7]);
          }
        }
      }
    };
    Cursor ci{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};  // the stage issued next
    tile_coords(ci);
    Cursor cs{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};  // the stage signalled next
    Cursor et{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};  // the tile drained next
    tile_coords(et);
    int ep_T = 0;
    bool ok = true;
    // drains tile ep_T (accumulator ep_T & 1) and frees the accumulator
    auto drain = [&]() -> bool {
      if (!wait(accf + (ep_T & 1), (ep_T >> 1) & 1)) return false;
      tc_fence_after();
      epilogue(et.tx, et.y, et.z, ep_T & 1);
      tc_fence_before();
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(acce + (ep_T & 1))) : "memory");
      ++ep_T;
      et.t += gridDim.x;
      if (et.t < ntiles32) tile_coords(et);
      return true;
    };
    for (int s = 0; s < nst32 + LAG && ok; ++s) {
      if (s < nst32) {
        // the buffer's previous stage must have been consumed
        if (s >= NS && !wait(empty + ci.buf, ci.par ^ 1)) {
          ok = false;
          break;
        }
        const int zz = ci.z + ci.st9 / 3 - 1, yy = ci.y + ci.st9 % 3 - 1, x0 = ci.tx * TC_M;
        const bool rowok = zz >= 0 && zz < D && yy >= 0 && yy < H;
        unsigned char *buf = sA + static_cast<size_t>(ci.buf) * SBY;
        const __nv_bfloat16 *row = X + ((static_cast<int64_t>(rowok ? zz : 0) * H + (rowok ? yy : 0)) * W + x0) * CIN;
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
          const int xx = x0 + u_x[j];
          const bool in = rowok && xx >= 0 && xx < W;
          const __nv_bfloat16 *src = in ? row + u_off[j] : X;
          if (u_dst[j] < 0) continue;
          if (!Mk) {
            cp_async16(buf + u_dst[j], src, in ? 16 : 0);
          } else {
            uint4 v = make_uint4(0, 0, 0, 0);
            if (in) {
              v = *reinterpret_cast<const uint4 *>(src);
              const uint4 mk = *reinterpret_cast<const uint4 *>(Mk + (src - X));
              __nv_bfloat16 *pv = reinterpret_cast<__nv_bfloat16 *>(&v);
              const __nv_bfloat16 *pm = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
              for (int q = 0; q < 8; ++q)
                if (!(__bfloat162float(pm[q]) > 0.0f)) pv[q] = __float2bfloat16(0.0f);
            }
            *reinterpret_cast<uint4 *>(buf + u_dst[j]) = v;
          }
        }
        advance(ci);
      }
      cp_async_commit();
      const int sd = s - LAG;
      if (sd >= 0) {
        // this thread's copies of stage sd have landed: hand them to the
        // async proxy and count them in
        cp_async_wait(LAG);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(full + cs.buf)) : "memory");
        advance(cs);
        // two stages of the next tile are handed over: drain the tile before
        if (sd == 9 * ep_T + 10 && !drain()) ok = false;
      }
    }
    while (ok && ep_T < my32) ok = drain();
    cp_async_wait(0);
  } else if (lane == 0) {
    // ------------------------------------------------------------ MMA warp
    Cursor cc{0, 0, 0, static_cast<int>(blockIdx.x), 0, 0, 0};
    int T = 0, last_buf = -1, last_par = 0;
    bool ok = true;
    for (int s = 0; s < nst32; ++s) {
      const int st9 = cc.st9, a = T & 1;
      if (st9 == 0 && T >= 2 && !wait(acce + a, ((T - 2) >> 1) & 1)) { ok = false; break; }
      if (!wait(full + cc.buf, cc.par)) { ok = false; break; }
      tc_fence_after();
      const int tapz = (st9 / 3) * 9 + (st9 % 3) * 3;
#pragma unroll 1
      for (int dxi = 0; dxi < 3; ++dxi)
        for (int kc = 0; kc < KC; ++kc) {
          const uint64_t ad =
              umma_smem_desc(smem_addr(sA + cc.buf * SBY + (2 * kc) * CV_PLANE + dxi * 16), CV_PLANE, 128);
          const uint64_t bd = umma_smem_desc(smem_addr(sB + ((tapz + dxi) * KC + kc) * bblk), 128, 256);
          mma_bf16(tmem + static_cast<uint32_t>(a) * ncols1, ad, bd, idesc, (st9 | dxi | kc) != 0 ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(empty + cc.buf))
                   : "memory");
      if (st9 == 8)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(accf + a))
                     : "memory");
      last_buf = cc.buf;
      last_par = cc.par;
      if (st9 == 8) ++T;
      advance(cc);
    }
    // after a failed wait, the MMAs in flight get one more bounded wait (the
    // last commit completes after all earlier ones) before TMEM is freed
    if (!ok && last_buf >= 0) mbar_wait(smem_addr(empty + last_buf), static_cast<uint32_t>(last_par));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// Instruction descriptor with both operands MN-major (bit 15: A, bit 16: B).
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int M, int N) {
  return umma_idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}

constexpr int WG_K = 32;  // voxels per stage of the weight gradient: two K = 16 MMAs

__host__ __device__ constexpr int wg_taps_per_tile(int Cin) { return 128 / Cin; }
__host__ __device__ constexpr int wg_mtiles(int Cin) { return (27 + 128 / Cin - 1) / (128 / Cin); }
__host__ __device__ constexpr size_t wg_smem_bytes(int Cin, int Cout) {
  return static_cast<size_t>(wg_mtiles(Cin)) * 2 * 4096 + static_cast<size_t>(2) * Cout * 32 + 64;
}
__host__ __device__ constexpr uint32_t wg_tmem_cols(int Cin, int Cout) {
  return wg_mtiles(Cin) * Cout <= 32 ? 32u : wg_mtiles(Cin) * Cout <= 64 ? 64u : wg_mtiles(Cin) * Cout <= 128 ? 128u
         : wg_mtiles(Cin) * Cout <= 256 ? 256u : 512u;
}

// Weight gradient dW[tap][ci][co] += sum_v X[v + tap][ci] G[v][co] (G = dY,
// or dY where Yo > 0) on tcgen05: D[m][n] = sum_k A[m][k] B[n][k] with
// m = (tap slot, ci), 128 / Cin taps per 128-row M tile (one TMEM
// accumulator of Cout columns per M tile), n = co, k = voxels, 32 voxels of
// one (z, y) row per stage.  For a fixed voxel both operands are contiguous
// along M or N (channels last), so A and B are MN-major: core matrices of 8
// voxels x 8 channels (16 bytes), K groups 128 bytes apart, 8-channel groups
// 256 bytes apart.  Persistent CTAs each sum a share of the voxels in TMEM
// and add their partial sums to dW with fp32 atomics at the end.
__global__ void __launch_bounds__(TC_THREADS, 1) wgrad_tc_kernel(
    const __nv_bfloat16 *__restrict__ X, const __nv_bfloat16 *__restrict__ dY, const __nv_bfloat16 *__restrict__ Yo,
    float *__restrict__ dW, int D, int H, int W, int Cin, int Cout) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int TPM = wg_taps_per_tile(Cin), MT = wg_mtiles(Cin);
  const int bblk = Cout * 32;
  unsigned char *sA = sm;                                  // [MT][2 k-steps] blocks of 4096 bytes
  unsigned char *sB = sm + static_cast<size_t>(MT) * 2 * 4096;  // [2 k-steps] blocks of Cout * 32 bytes
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sB + 2 * bblk);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = wg_tmem_cols(Cin, Cout);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16_mn(TC_M, Cout);
  const uint32_t bar_a = smem_addr(bar);
  uint32_t phase = 0;
  bool ok = true, any = false;
  const int nxc = (W + WG_K - 1) / WG_K;
  const int64_t nchunks = static_cast<int64_t>(D) * H * nxc;
  const int cg_in = Cin / 8, cg_out = Cout / 8;
  // 32-bit chunk arithmetic (the host rejects grids with more chunks)
  for (int t = blockIdx.x; t < static_cast<int>(nchunks) && ok; t += gridDim.x) {
    const int xc = t % nxc;
    const int zy = t / nxc;
    const int y = zy % H, z = zy / H;
    const int x0 = xc * WG_K;
    // B: G of the chunk's 32 voxels, 8 output channels per unit
    for (int i = tid; i < WG_K * cg_out; i += TC_THREADS) {
      const int k = i % WG_K, g = i / WG_K;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (x0 + k < W) {
        const int64_t off = ((static_cast<int64_t>(z) * H + y) * W + x0 + k) * Cout + g * 8;
        v = *reinterpret_cast<const uint4 *>(dY + off);
        if (Yo) {
          const uint4 mk = *reinterpret_cast<const uint4 *>(Yo + off);
          __nv_bfloat16 *pv = reinterpret_cast<__nv_bfloat16 *>(&v);
          const __nv_bfloat16 *pm = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (!(__bfloat162float(pm[q]) > 0.0f)) pv[q] = __float2bfloat16(0.0f);
        }
      }
      const int ks = k >> 4, kk = k & 15;
      *reinterpret_cast<uint4 *>(sB + ks * bblk + g * 256 + (kk >> 3) * 128 + (kk & 7) * 16) = v;
    }
    // A: the shifted inputs of the taps of every M tile, 8 input channels per unit
    for (int i = tid; i < MT * TPM * cg_in * WG_K; i += TC_THREADS) {
      const int k = i % WG_K;
      int r = i / WG_K;
      const int cg = r % cg_in;
      r /= cg_in;
      const int slot = r % TPM, mt = r / TPM;
      const int tap = mt * TPM + slot;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (tap < 27 && x0 + k < W) {
        const int zz = z + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, xx = x0 + k + tap % 3 - 1;
        if (zz >= 0 && zz < D && yy >= 0 && yy < H && xx >= 0 && xx < W)
          v = *reinterpret_cast<const uint4 *>(X + ((static_cast<int64_t>(zz) * H + yy) * W + xx) * Cin + cg * 8);
      }
      const int mg = slot * cg_in + cg;  // 8-row group of m = slot * Cin + 8 cg
      const int ks = k >> 4, kk = k & 15;
      *reinterpret_cast<uint4 *>(sA + (mt * 2 + ks) * 4096 + mg * 256 + (kk >> 3) * 128 + (kk & 7) * 16) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      for (int mt = 0; mt < MT; ++mt)
        for (int ks = 0; ks < 2; ++ks) {
          const uint64_t a = umma_smem_desc(smem_addr(sA + (mt * 2 + ks) * 4096), 128, 256);
          const uint64_t b = umma_smem_desc(smem_addr(sB + ks * bblk), 128, 256);
          mma_bf16(tmem + static_cast<uint32_t>(mt * Cout), a, b, idesc, (any || ks) ? 1u : 0u);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                   : "memory");
    }
    ok = __syncthreads_and(mbar_wait(bar_a, phase) ? 1 : 0) != 0;
    phase ^= 1u;
    tc_fence_after();
    any = true;
  }
  if (ok && any) {
    // partial sums: warp w holds rows m = 32w..32w+31 of every M tile
    const int m = warp * 32 + lane, slot = m / Cin, ci = m % Cin;
    for (int mt = 0; mt < MT; ++mt) {
      const int tap = mt * TPM + slot;
      for (int c0 = 0; c0 < Cout; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(mt * Cout + c0), r);
        if (tap < 27) {
          float *dst = dW + (static_cast<int64_t>(tap) * Cin + ci) * Cout + c0;
#pragma unroll
          for (int j = 0; j < 16; ++j) atomicAdd(dst + j, __uint_as_float(r[j]));
        }
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(&g_tc_err, 1);
    mbar_wait(bar_a, phase ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// db[co] += sum_v G[v][co] (G = dY, or dY where Yo > 0): one block per
// chunk of voxels, per-thread channel sums, one atomic per channel and block.
__global__ void bias_sum_kernel(const __nv_bfloat16 *__restrict__ dY, const __nv_bfloat16 *__restrict__ Yo,
                                float *__restrict__ db, int64_t nvox, int Cout) {
  extern __shared__ float s_db[];
  for (int c = threadIdx.x; c < Cout; c += blockDim.x) s_db[c] = 0.0f;
  __syncthreads();
  const int per = blockDim.x / Cout;  // voxels in flight per block step
  const int co = threadIdx.x % Cout, lane_v = threadIdx.x / Cout;
  float acc = 0.0f;
  if (lane_v < per)
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * per + lane_v; v < nvox; v += static_cast<int64_t>(gridDim.x) * per) {
      const int64_t o = v * Cout + co;
      const float g = __bfloat162float(dY[o]);
      acc += (!Yo || __bfloat162float(Yo[o]) > 0.0f) ? g : 0.0f;
    }
  if (lane_v < per) atomicAdd(&s_db[co], acc);
  __syncthreads();
  for (int c = threadIdx.x; c < Cout; c += blockDim.x) atomicAdd(&db[c], s_db[c]);
}

}  // namespace

using namespace orsp;

extern "C" int orsp_warm_conv3d_tc(const void *X, const void *mask, const void *Wt, const float *bias, void *Y,
                                   float *Yf, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                                   int32_t relu, uintptr_t stream) {
  if (!X || !Wt || (!Y && !Yf) || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cin % 16 || Cout <= 0 ||
      Cout % 16 || Cout > 64) {
    set_error("warm_conv3d_tc: bad arguments (Cin, Cout multiples of 16, Cout <= 64)");
    return ORSP_ERR_ARG;
  }
  const int ns = cv_stages(Cin, Cout);
  if (ns < 2) {
    set_error("warm_conv3d_tc: weights of this Cin x Cout and two stages do not fit in shared memory");
    return ORSP_ERR_ARG;
  }
  const size_t smem = cv_smem_bytes(Cin, Cout, ns);
  int dev = 0, sms = 0;
  ORSP_CUDA(cudaGetDevice(&dev));
  ORSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  void (*kfn)(const __nv_bfloat16 *, const __nv_bfloat16 *, const __nv_bfloat16 *, const float *, __nv_bfloat16 *,
              float *, int, int, int, int, int, int, int) =
      Cin == 16 ? conv3d_tc_kernel<2> : Cin == 32 ? conv3d_tc_kernel<4> : Cin == 64 ? conv3d_tc_kernel<8> : nullptr;
  if (!kfn) {
    set_error("warm_conv3d_tc: Cin must be 16, 32 or 64");
    return ORSP_ERR_ARG;
  }
  ORSP_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t ntiles = static_cast<int64_t>(D) * H * ((W + TC_M - 1) / TC_M);
  if (ntiles * 9 > INT32_MAX) {
    set_error("warm_conv3d_tc: grid too large (the stage counters are 32-bit)");
    return ORSP_ERR_ARG;
  }
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ntiles, sms)));
  // the warp-specialised kernel (producer warps and an MMA warp handing
  // stages over through mbarriers); ORSP_WARM_TC_WS=0: the kernel with one
  // block barrier per stage
  const char *ws = getenv("ORSP_WARM_TC_WS");
  if (!(ws && ws[0] == '0')) {
    decltype(kfn) kws = Cin == 16 ? conv3d_tc_ws_kernel<2> : Cin == 32 ? conv3d_tc_ws_kernel<4>
                                                                       : conv3d_tc_ws_kernel<8>;
    const size_t smem_ws = ws_smem_bytes(Cin, Cout, ns);
    ORSP_CUDA(cudaFuncSetAttribute(kws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_ws));
    kws<<<grid, WS_THREADS, smem_ws, (cudaStream_t)stream>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)mask,
                                                             (const __nv_bfloat16 *)Wt, bias, (__nv_bfloat16 *)Y, Yf,
                                                             D, H, W, Cin, Cout, relu, ns);
    ORSP_CUDA(cudaGetLastError());
    return ORSP_OK;
  }
  kfn<<<grid, CV_THREADS, smem, (cudaStream_t)stream>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)mask,
                                                        (const __nv_bfloat16 *)Wt, bias, (__nv_bfloat16 *)Y, Yf, D, H,
                                                        W, Cin, Cout, relu, ns);
  ORSP_CUDA(cudaGetLastError());
  return ORSP_OK;
}

extern "C" int orsp_warm_tc_status(int32_t *expired) {
  if (!expired) { set_error("warm_tc_status: NULL argument"); return ORSP_ERR_ARG; }
  int v = 0, zero = 0;
  ORSP_CUDA(cudaMemcpyFromSymbol(&v, g_tc_err, sizeof(int)));
  ORSP_CUDA(cudaMemcpyToSymbol(g_tc_err, &zero, sizeof(int)));
  *expired = v;
  return ORSP_OK;
}

extern "C" int orsp_warm_wgrad_tc(const void *X, const void *dY, const void *Yo, float *dW, float *db, int32_t D,
                                  int32_t H, int32_t W, int32_t Cin, int32_t Cout, uintptr_t stream) {
  if (!X || !dY || !dW || D <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cin % 16 || Cin > 64 || Cout <= 0 ||
      Cout % 16 || Cout > 64 || wg_mtiles(Cin) * Cout > 512) {
    set_error("warm_wgrad_tc: bad arguments (Cin, Cout multiples of 16, at most 64, accumulators within TMEM)");
    return ORSP_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t smem = wg_smem_bytes(Cin, Cout);
  int dev = 0, sms = 0;
  ORSP_CUDA(cudaGetDevice(&dev));
  ORSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ORSP_CUDA(cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t nchunks = static_cast<int64_t>(D) * H * ((W + WG_K - 1) / WG_K);
  if (nchunks > INT32_MAX) {
    set_error("warm_wgrad_tc: grid too large (the chunk counter is 32-bit)");
    return ORSP_ERR_ARG;
  }
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(nchunks, sms)));
  wgrad_tc_kernel<<<grid, TC_THREADS, smem, st>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)dY,
                                                  (const __nv_bfloat16 *)Yo, dW, D, H, W, Cin, Cout);
  ORSP_CUDA(cudaGetLastError());
  if (db) {
    const int64_t nvox = static_cast<int64_t>(D) * H * W;
    const int threads = (256 / Cout) * Cout;
    const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((nvox + 255) / 256, sms * 8)));
    bias_sum_kernel<<<blocks, threads, Cout * sizeof(float), st>>>((const __nv_bfloat16 *)dY,
                                                                   (const __nv_bfloat16 *)Yo, db, nvox, Cout);
    ORSP_CUDA(cudaGetLastError());
  }
  return ORSP_OK;
}
