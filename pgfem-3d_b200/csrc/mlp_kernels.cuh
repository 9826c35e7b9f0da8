// mlp_kernels.cuh -- the warm-start network of the crystal-plasticity local
// Newton on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// No counterpart in the reference: PGFem3D starts the CP Newton from the
// elastic predictor (src/plasticity_model.cc:1148-1224).  The network maps 34
// per-point features (incremental F, pF_n, 12 slip resistances, lattice
// quaternion) through three GELU layers of width 128 to the 12 slip
// increments dt*gamma_dot_a; its prediction only seeds the FP64 Newton.
//
// Arithmetic: BF16 operands, FP32 accumulation in tensor memory (TMEM),
// biases and GELU in FP32.  One CTA of 4 warps owns a tile of 128 points; the
// tile is the M = 128 dimension of every forward GEMM, each layer is ONE
// tcgen05.mma chain (K/16 instructions of M128 x N128 x K16) issued by a
// single thread, completion tracked by tcgen05.commit on an mbarrier, and the
// epilogue reads the accumulator rows back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = tile rows).
//
// Shared-memory operand layout: every matrix (weights, activations, error
// terms) is stored as 8x8 BF16 core matrices (128 contiguous bytes, rows of
// 16 bytes), core matrices row-group major:
//     elem(r, c) at ((r/8)*(C/8) + c/8)*64 + (r%8)*8 + c%8.
// The same bytes serve as a K-major operand (rows = M or N index, columns =
// K index: LBO = 128 B between K groups, SBO = C/8*128 B between row groups)
// or as an MN-major operand (rows = K index, columns = M or N index: LBO =
// C/8*128 B, SBO = 128 B), so the backward GEMMs (dW = dZ^T H, dH = dZ W)
// read the forward operands in place, with no transposed copies.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pgb {
namespace mlp {

constexpr int kIn = 34, kInP = 48, kH = 128, kOut = 12, kOutP = 16, kTile = 128, kThreads = 128;
// FP32 master parameter vector: W1[128][34] b1 W2[128][128] b2 W3 b3 W4[12][128] b4
constexpr int oW1 = 0, ob1 = oW1 + kH * kIn, oW2 = ob1 + kH, ob2 = oW2 + kH * kH, oW3 = ob2 + kH,
              ob3 = oW3 + kH * kH, oW4 = ob3 + kH, ob4 = oW4 + kOut * kH, kNParam = ob4 + kOut;
// padded BF16 weights, row-major [out][in]: W1 [128][48], W2, W3 [128][128], W4 [16][128]
constexpr int pW1 = 0, pW2 = pW1 + kH * kInP, pW3 = pW2 + kH * kH, pW4 = pW3 + kH * kH,
              kNPW = pW4 + kOutP * kH;
// padded FP32 biases
constexpr int pb1 = 0, pb2 = 128, pb3 = 256, pb4 = 384, kNPB = 400;
// feature / target scaling: x_mean[34], 1/x_std[34], y_std[12]
constexpr int kScale = 80;

// shared-memory byte offsets (all multiples of 128)
constexpr uint32_t sW1 = 0, sW2 = sW1 + kH * kInP * 2, sW3 = sW2 + kH * kH * 2, sW4 = sW3 + kH * kH * 2,
                   sX0 = sW4 + kOutP * kH * 2, sH1 = sX0 + kTile * kInP * 2;
// inference: one activation buffer reused layer to layer
constexpr uint32_t sInfBias = sH1 + kTile * kH * 2, sInfScale = sInfBias + kNPB * 4,
                   sInfMisc = sInfScale + kScale * 4, kInfSmem = sInfMisc + 64;
// training: H1, H2, H3 kept for the weight gradients, one error-term buffer
constexpr uint32_t sH2 = sH1 + kTile * kH * 2, sH3 = sH2 + kTile * kH * 2, sDZ = sH3 + kTile * kH * 2,
                   sTrBias = sDZ + kTile * kH * 2, sTrScale = sTrBias + kNPB * 4,
                   sTrMisc = sTrScale + kScale * 4, kTrainSmem = sTrMisc + 64;
static_assert(kTrainSmem <= 232448, "training tile exceeds the 227 KB shared-memory limit");

struct MlpDev {
  const __nv_bfloat16 *w;  // kNPW
  const float *b;          // kNPB
  const float *scale;      // kScale
  unsigned *err;           // bit 0: an mbarrier wait ran out
  uint64_t wait_ns;        // bound of every mbarrier wait
  int stall;               // test of the failure path: the first tile's first MMA chain is not issued
};

constexpr uint64_t kWaitNs = 2000000000ull;  // default bound of every mbarrier wait (2 s)

// ---------------------------------------------------------------- helpers --

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// UMMA shared-memory descriptor, no swizzle (canonical interleaved layout):
// start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46), version 1 [46,48),
// base offset 0, layout type SWIZZLE_NONE (0) [61,64).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// A/B major (0 = K-major, 1 = MN-major), N >> 3 at [17,23), M >> 4 at [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct Opnd {
  uint32_t addr, lbo, sbo;
};
// matrix of `cols` columns stored as core matrices, used with K along columns
__device__ __forceinline__ Opnd kmajor(uint32_t addr, int cols) { return {addr, 128u, (uint32_t)cols * 16u}; }
// ... used with K along rows
__device__ __forceinline__ Opnd mnmajor(uint32_t addr, int cols) { return {addr, (uint32_t)cols * 16u, 128u}; }

// D[tmem] (+)= A * B^T over `ksteps` K-slices of 16; issued by one thread.
__device__ __forceinline__ void mma_chain(uint32_t d_tmem, Opnd A, Opnd B, int ksteps, uint32_t idesc) {
  for (int k = 0; k < ksteps; k++) {
    const uint64_t ad = sdesc(A.addr + 2u * (uint32_t)k * A.lbo, A.lbo, A.sbo);
    const uint64_t bd = sdesc(B.addr + 2u * (uint32_t)k * B.lbo, B.lbo, B.sbo);
    const uint32_t acc = k > 0 ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
  }
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor-core (async) proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the completion of phase `parity`; false after `limit` ns.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, uint64_t limit) {
  const uint64_t t0 = gtimer();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (gtimer() - t0 > limit) return false;
  }
}

// whole warp: allocate `ncols` TMEM columns, address written to shared `slot`
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane; the
// wait is tied to the destination registers so no use can move above it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7, r8, r9, r10, r11, r12, r13, r14, r15;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7), "=r"(r8), "=r"(r9),
        "=r"(r10), "=r"(r11), "=r"(r12), "=r"(r13), "=r"(r14), "=r"(r15)
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7), "+r"(r8),
                 "+r"(r9), "+r"(r10), "+r"(r11), "+r"(r12), "+r"(r13), "+r"(r14), "+r"(r15)::"memory");
  v[0] = __uint_as_float(r0), v[1] = __uint_as_float(r1), v[2] = __uint_as_float(r2);
  v[3] = __uint_as_float(r3), v[4] = __uint_as_float(r4), v[5] = __uint_as_float(r5);
  v[6] = __uint_as_float(r6), v[7] = __uint_as_float(r7), v[8] = __uint_as_float(r8);
  v[9] = __uint_as_float(r9), v[10] = __uint_as_float(r10), v[11] = __uint_as_float(r11);
  v[12] = __uint_as_float(r12), v[13] = __uint_as_float(r13), v[14] = __uint_as_float(r14);
  v[15] = __uint_as_float(r15);
}

// byte offset of the 16-byte row segment (r, c0..c0+7) of a blocked matrix with C columns
__device__ __forceinline__ uint32_t blk_off(int r, int c0, int C) {
  return (uint32_t)((((r >> 3) * (C >> 3) + (c0 >> 3)) * 64 + (r & 7) * 8) * 2);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
// store 8 floats as BF16 at (r, c0..c0+7)
__device__ __forceinline__ void st8(unsigned char *base, int r, int c0, int C, const float *v) {
  uint4 q;
  q.x = pack2(v[0], v[1]);
  q.y = pack2(v[2], v[3]);
  q.z = pack2(v[4], v[5]);
  q.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(base + blk_off(r, c0, C)) = q;
}
__device__ __forceinline__ float ld_blk(const unsigned char *base, int r, int c, int C) {
  const __nv_bfloat16 *p = reinterpret_cast<const __nv_bfloat16 *>(base + blk_off(r, c & ~7, C));
  return __bfloat162float(p[c & 7]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// row-major padded global BF16 matrix R x C -> blocked shared layout
__device__ __forceinline__ void load_blocked(unsigned char *dst, const __nv_bfloat16 *src, int R, int C) {
  const int chunks = R * C / 8;
  for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
    const int r = i / (C / 8), cg = i % (C / 8);
    *reinterpret_cast<uint4 *>(dst + blk_off(r, cg * 8, C)) = reinterpret_cast<const uint4 *>(src)[i];
  }
}

__device__ __forceinline__ void load_params(unsigned char *sm, const MlpDev &m, float *sb, float *ss) {
  load_blocked(sm + sW1, m.w + pW1, kH, kInP);
  load_blocked(sm + sW2, m.w + pW2, kH, kH);
  load_blocked(sm + sW3, m.w + pW3, kH, kH);
  load_blocked(sm + sW4, m.w + pW4, kOutP, kH);
  for (int i = threadIdx.x; i < kNPB; i += blockDim.x) sb[i] = m.b[i];
  for (int i = threadIdx.x; i < kScale; i += blockDim.x) ss[i] = m.scale[i];
}

// one normalised feature row (34 + zero padding to 48) of tile row r
__device__ __forceinline__ void load_x_row(unsigned char *sX, int r, const float *xrow, const float *ss) {
  float v[kInP];
#pragma unroll
  for (int j = 0; j < kInP; j++) v[j] = (xrow && j < kIn) ? (xrow[j] - ss[j]) * ss[kIn + j] : 0.0f;
#pragma unroll
  for (int c = 0; c < kInP; c += 8) st8(sX, r, c, kInP, v + c);
}

// hidden-layer epilogue: rows of this thread, H = GELU(Z + b) -> blocked BF16
__device__ __forceinline__ void epi_hidden(uint32_t tz, unsigned char *sHout, int r, const float *bias) {
#pragma unroll 1
  for (int c0 = 0; c0 < kH; c0 += 16) {
    float v[16];
    tmem_ld16(tz + (uint32_t)c0, v);
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = gelu(v[i] + bias[c0 + i]);
    st8(sHout, r, c0, kH, v);
    st8(sHout, r, c0 + 8, kH, v + 8);
  }
}

// ------------------------------------------------------------- inference --
// Persistent over tiles of 128 points: y[n][12] = network(x[n][34]) in raw units.
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_forward(const MlpDev m, long n, const float *__restrict__ x, float *__restrict__ y) {
  extern __shared__ __align__(128) unsigned char sm[];
  float *sb = reinterpret_cast<float *>(sm + sInfBias);
  float *ss = reinterpret_cast<float *>(sm + sInfScale);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + sInfMisc);
  uint32_t *slot = reinterpret_cast<uint32_t *>(sm + sInfMisc + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ab = smem_u32(sm), mb = smem_u32(mbar);
  if (warp == 0) tmem_alloc(smem_u32(slot), 128);
  if (tid == 0) mbar_init(mb, 1);
  load_params(sm, m, sb, ss);
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tbase = *slot;
  const uint32_t tme = tbase + ((uint32_t)(warp * 32) << 16);  // this warp's lane quarter, column 0
  const long ntiles = (n + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool fail = false;
  constexpr uint32_t ID_H = idesc_bf16(128, kH, 0, 0), ID_O = idesc_bf16(128, kOutP, 0, 0);
  for (long t = blockIdx.x; t < ntiles && !fail; t += gridDim.x) {
    const long row = t * kTile + tid;
    load_x_row(sm + sX0, tid, row < n ? x + row * kIn : nullptr, ss);
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    for (int l = 0; l < 4 && !fail; l++) {
      // (with m.stall the CTA's first chain and its commit are not issued: the
      // wait below runs out with no MMA in flight)
      if (tid == 0 && !(m.stall && l == 0 && t == blockIdx.x)) {
        if (l == 0)
          mma_chain(tbase, kmajor(ab + sX0, kInP), kmajor(ab + sW1, kInP), kInP / 16, ID_H);
        else if (l < 3)
          mma_chain(tbase, kmajor(ab + sH1, kH), kmajor(ab + (l == 1 ? sW2 : sW3), kH), kH / 16, ID_H);
        else
          mma_chain(tbase, kmajor(ab + sH1, kH), kmajor(ab + sW4, kH), kH / 16, ID_O);
        mma_commit(mb);
      }
      const bool ok = mbar_wait(mb, phase, m.wait_ns);
      phase ^= 1;
      if (__syncthreads_or(!ok)) {
        fail = true;
        break;
      }
      tc_after();
      if (l < 3) {
        epi_hidden(tme, sm + sH1, tid, sb + (l == 0 ? pb1 : l == 1 ? pb2 : pb3));
      } else {
        float v[16];
        tmem_ld16(tme, v);  // warp-wide: every lane loads, rows past n store nothing
        if (row < n) {
#pragma unroll
          for (int i = 0; i < kOut; i++) y[row * kOut + i] = (v[i] + sb[pb4 + i]) * ss[2 * kIn + i];
        }
      }
      fence_async_smem();
      tc_before();
      __syncthreads();
      tc_after();
    }
  }
  if (fail) {
    mbar_wait(mb, phase ^ 1u, m.wait_ns);  // bounded: let a late MMA finish before its TMEM is released
    if (tid == 0) atomicOr(m.err, 1u);
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (warp == 0) tmem_free(tbase, 128);
}

// -------------------------------------------------------------- training --
// One tile of 128 samples (rows perm[first + i] of x/t, i < count): forward,
// loss 1/(2B) sum (out - t/y_std)^2, backward; parameter gradients added to
// grad (FP32, master layout), loss added to *loss.
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_train(const MlpDev m, long count, long first, const int *__restrict__ perm,
                const float *__restrict__ x, const float *__restrict__ tg, float inv_batch,
                float *__restrict__ grad, double *__restrict__ loss) {
  extern __shared__ __align__(128) unsigned char sm[];
  float *sb = reinterpret_cast<float *>(sm + sTrBias);
  float *ss = reinterpret_cast<float *>(sm + sTrScale);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + sTrMisc);
  uint32_t *slot = reinterpret_cast<uint32_t *>(sm + sTrMisc + 8);
  double *red = reinterpret_cast<double *>(sm + sTrMisc + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ab = smem_u32(sm), mb = smem_u32(mbar);
  if (warp == 0) tmem_alloc(smem_u32(slot), 512);
  if (tid == 0) mbar_init(mb, 1);
  load_params(sm, m, sb, ss);
  __syncthreads();  // the feature scaling in ss is read by every row below
  const long i_row = (long)blockIdx.x * kTile + tid;
  const bool valid = i_row < count;
  const long src = valid ? (perm ? (long)perm[first + i_row] : first + i_row) : 0;
  load_x_row(sm + sX0, tid, valid ? x + src * kIn : nullptr, ss);
  fence_async_smem();
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tbase = *slot;
  const uint32_t lq = (uint32_t)(warp * 32) << 16;
  // TMEM columns: Z1 [0,128) Z2 [128,256) Z3 [256,384) scratch S [384,512)
  const uint32_t cZ1 = 0, cZ2 = 128, cZ3 = 256, cS = 384;
  uint32_t phase = 0;
  bool fail = false;
  constexpr uint32_t ID_KK = idesc_bf16(128, kH, 0, 0), ID_KK_O = idesc_bf16(128, kOutP, 0, 0);
  constexpr uint32_t ID_MM_O = idesc_bf16(128, kOutP, 1, 1), ID_MM = idesc_bf16(128, kH, 1, 1);
  constexpr uint32_t ID_MM_IN = idesc_bf16(128, kInP, 1, 1), ID_KM = idesc_bf16(128, kH, 0, 1);
  auto sync_all = [&]() {
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
  };
  auto wait_mma = [&]() -> bool {
    const bool ok = mbar_wait(mb, phase, m.wait_ns);
    phase ^= 1;
    if (__syncthreads_or(!ok)) return false;
    tc_after();
    return true;
  };
  auto bias_grad = [&](int C, int nvalid, int og) {
    __syncthreads();
    if (tid < nvalid) {
      float s = 0.0f;
      for (int r = 0; r < kTile; r++) s += ld_blk(sm + sDZ, r, tid, C);
      atomicAdd(grad + og + tid, s);
    }
  };
  // dW rows: this thread's TMEM lane = output neuron `tid`, columns = inputs
  auto dw_rows = [&](uint32_t col, int kvalid, int ow) {
    for (int c0 = 0; c0 < (kvalid + 15) / 16 * 16; c0 += 16) {
      float v[16];
      tmem_ld16(tbase + lq + col + (uint32_t)c0, v);
#pragma unroll
      for (int i = 0; i < 16; i++)
        if (c0 + i < kvalid) atomicAdd(grad + ow + tid * kvalid + c0 + i, v[i]);
    }
  };
  // dZ_l = (dH . W_{l+1}) * GELU'(Z_l + b_l) -> sDZ (blocked BF16, 128 columns)
  auto epi_dz = [&](uint32_t cz, const float *bias) {
    for (int c0 = 0; c0 < kH; c0 += 16) {
      float dh[16], z[16];
      tmem_ld16(tbase + lq + cS + (uint32_t)c0, dh);
      tmem_ld16(tbase + lq + cz + (uint32_t)c0, z);
#pragma unroll
      for (int i = 0; i < 16; i++) dh[i] = valid ? dh[i] * gelu_d(z[i] + bias[c0 + i]) : 0.0f;
      st8(sm + sDZ, tid, c0, kH, dh);
      st8(sm + sDZ, tid, c0 + 8, kH, dh + 8);
    }
  };
  do {
    // forward
    const uint32_t sHs[3] = {sH1, sH2, sH3}, sWs[3] = {sW1, sW2, sW3}, cZs[3] = {cZ1, cZ2, cZ3};
    for (int l = 0; l < 3 && !fail; l++) {
      if (tid == 0) {
        if (l == 0)
          mma_chain(tbase + cZ1, kmajor(ab + sX0, kInP), kmajor(ab + sW1, kInP), kInP / 16, ID_KK);
        else
          mma_chain(tbase + cZs[l], kmajor(ab + sHs[l - 1], kH), kmajor(ab + sWs[l], kH), kH / 16, ID_KK);
        mma_commit(mb);
      }
      if (!wait_mma()) {
        fail = true;
        break;
      }
      epi_hidden(tbase + lq + cZs[l], sm + sHs[l], tid, sb + (l == 0 ? pb1 : l == 1 ? pb2 : pb3));
      sync_all();
    }
    if (fail) break;
    if (tid == 0) {
      mma_chain(tbase + cS, kmajor(ab + sH3, kH), kmajor(ab + sW4, kH), kH / 16, ID_KK_O);
      mma_commit(mb);
    }
    if (!wait_mma()) {
      fail = true;
      break;
    }
    {  // output error terms dZ4 = (out - t/y_std) / B -> sDZ as a 128 x 16 matrix
      float v[16];
      tmem_ld16(tbase + lq + cS, v);
      double l2 = 0.0;
#pragma unroll
      for (int i = 0; i < 16; i++) {
        float r = 0.0f;
        if (valid && i < kOut) {
          r = (v[i] + sb[pb4 + i]) - tg[src * kOut + i] / ss[2 * kIn + i];
          l2 += (double)r * (double)r;
        }
        v[i] = r * inv_batch;
      }
      st8(sm + sDZ, tid, 0, kOutP, v);
      st8(sm + sDZ, tid, 8, kOutP, v + 8);
      for (int o = 16; o; o >>= 1) l2 += __shfl_xor_sync(0xffffffffu, l2, o);
      if (lane == 0) red[warp] = l2;
    }
    sync_all();
    if (tid == 0) {
      atomicAdd(loss, 0.5 * (red[0] + red[1] + red[2] + red[3]) * (double)inv_batch);
      // dW4^T [k][n] = H3^T dZ4 : M = 128 (k), N = 16 (n), K = samples
      mma_chain(tbase + cS, mnmajor(ab + sH3, kH), mnmajor(ab + sDZ, kOutP), kTile / 16, ID_MM_O);
      mma_commit(mb);
    }
    bias_grad(kOutP, kOut, ob4);
    if (!wait_mma()) {
      fail = true;
      break;
    }
    {
      float v[16];
      tmem_ld16(tbase + lq + cS, v);
#pragma unroll
      for (int i = 0; i < kOut; i++) atomicAdd(grad + oW4 + i * kH + tid, v[i]);
    }
    sync_all();
    if (tid == 0) {  // dH3 = dZ4 W4 : M = samples, N = 128, K = 16
      mma_chain(tbase + cS, kmajor(ab + sDZ, kOutP), mnmajor(ab + sW4, kH), 1, ID_KM);
      mma_commit(mb);
    }
    if (!wait_mma()) {
      fail = true;
      break;
    }
    epi_dz(cZ3, sb + pb3);
    sync_all();
    // layers 3, 2: dW_l = dZ_l^T H_{l-1} into Z_l's columns, dH_{l-1} = dZ_l W_l into S
    const uint32_t sHprev[2] = {sH2, sH1}, sWl[2] = {sW3, sW2}, cZl[2] = {cZ3, cZ2}, cZprev[2] = {cZ2, cZ1};
    const int obias[2] = {ob3, ob2}, ow[2] = {oW3, oW2}, pbp[2] = {pb2, pb1};
    for (int j = 0; j < 2 && !fail; j++) {
      if (tid == 0) {
        mma_chain(tbase + cZl[j], mnmajor(ab + sDZ, kH), mnmajor(ab + sHprev[j], kH), kTile / 16, ID_MM);
        mma_chain(tbase + cS, kmajor(ab + sDZ, kH), mnmajor(ab + sWl[j], kH), kH / 16, ID_KM);
        mma_commit(mb);
      }
      bias_grad(kH, kH, obias[j]);
      if (!wait_mma()) {
        fail = true;
        break;
      }
      dw_rows(cZl[j], kH, ow[j]);
      __syncthreads();
      epi_dz(cZprev[j], sb + pbp[j]);
      sync_all();
    }
    if (fail) break;
    if (tid == 0) {  // dW1 = dZ1^T X0 : M = 128, N = 48, K = samples
      mma_chain(tbase + cZ1, mnmajor(ab + sDZ, kH), mnmajor(ab + sX0, kInP), kTile / 16, ID_MM_IN);
      mma_commit(mb);
    }
    bias_grad(kH, kH, ob1);
    if (!wait_mma()) {
      fail = true;
      break;
    }
    dw_rows(cZ1, kIn, oW1);
  } while (false);
  if (fail) {
    mbar_wait(mb, phase ^ 1u, m.wait_ns);  // bounded: let a late MMA finish before its TMEM is released
    if (tid == 0) atomicOr(m.err, 1u);
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (warp == 0) tmem_free(tbase, 512);
}

// Adam on the FP32 master vector; re-packs the BF16 weights / FP32 biases and
// clears the gradient for the next step.
__global__ void k_mlp_adam(float *__restrict__ p, float *__restrict__ g, float *__restrict__ mo,
                           float *__restrict__ ve, __nv_bfloat16 *__restrict__ w, float *__restrict__ b,
                           float lr, float b1, float b2, float eps, float c1, float c2, int update) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNParam) return;
  float v = p[i];
  if (update) {
    const float gi = g[i];
    const float m1 = b1 * mo[i] + (1.0f - b1) * gi;
    const float v1 = b2 * ve[i] + (1.0f - b2) * gi * gi;
    mo[i] = m1;
    ve[i] = v1;
    v -= lr * (m1 * c1) / (sqrtf(v1 * c2) + eps);
    p[i] = v;
    g[i] = 0.0f;
  }
  if (i < ob1) w[pW1 + (i / kIn) * kInP + i % kIn] = __float2bfloat16_rn(v);
  else if (i < oW2) b[pb1 + i - ob1] = v;
  else if (i < ob2) w[pW2 + i - oW2] = __float2bfloat16_rn(v);
  else if (i < oW3) b[pb2 + i - ob2] = v;
  else if (i < ob3) w[pW3 + i - oW3] = __float2bfloat16_rn(v);
  else if (i < oW4) b[pb3 + i - ob3] = v;
  else if (i < ob4) w[pW4 + i - oW4] = __float2bfloat16_rn(v);
  else b[pb4 + i - ob4] = v;
}

// per-column sum and sum of squares (FP64) of a row-major n x NC FP32 array
template <int NC>
__global__ void k_col_stats(const float *__restrict__ x, long n, double *__restrict__ acc) {
  double s[NC], q[NC];
#pragma unroll
  for (int j = 0; j < NC; j++) s[j] = q[j] = 0.0;
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < NC; j++) {
      const double v = x[r * NC + j];
      s[j] += v;
      q[j] += v * v;
    }
  }
#pragma unroll
  for (int j = 0; j < NC; j++) {
    double a = s[j], c = q[j];
    for (int o = 16; o; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(acc + j, a);
      atomicAdd(acc + NC + j, c);
    }
  }
}

}  // namespace mlp
}  // namespace pgb
