// Learned-closure inference on the 5th-generation tensor cores (tcgen05, sm_100a):
// 128-cell tiles, BF16 operands staged in shared memory in the K-major interleaved
// (no swizzle) canonical layout, FP32 accumulators in tensor memory (TMEM).
//
// Per tile of 128 cells (row r of every matrix = cell r = TMEM lane r):
//   D1[128 x 32] = A1[128 x 16] B1^T     A1 = the 8 inputs, K padded to 16
//   D2[128 x 32] = A2[128 x 32] B2^T     A2 = GELU(D1 + b1), BF16
//   D3[128 x 16] = A2'[128 x 32] B3^T    A2' = GELU(D2 + b2), column 0 of D3 + b3 -> softplus
// One thread issues each layer's MMAs and commits them to an mbarrier; every warp then
// reads its 32 TMEM lanes (tcgen05.ld 32x32b), applies bias and activation and writes the
// next layer's A operand.  Descriptor fields follow the SM100 UMMA definitions:
//   shared-memory descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
//     version 1 [46,48), base offset 0, layout type 0 (no swizzle) [61,64);
//   instruction descriptor (kind::f16): D F32 [4,6) = 1, A BF16 [7,10) = 1, B BF16
//     [10,13) = 1, both K-major, N >> 3 [17,23), M >> 4 [24,29).
#pragma once
#include "sgs_mlp.cuh"

namespace aerosim {

constexpr int kUmmaRows = 128;
// Byte offset of element (r, k) of a K-major operand with K columns: core matrices of
// 8 rows x 16 bytes; K-adjacent core matrices 128 B apart (LBO), 8-row groups
// K / 8 x 128 B apart (SBO).
__host__ __device__ constexpr uint32_t umma_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// Shared-memory image of the weights (B operands, N rows x K): W1 32 x 16 (K padded),
// W2 32 x 32, W3 16 x 32 (row 0 = W3, rows 1..15 zero).
constexpr int kUmmaB1 = 0, kUmmaB2 = 32 * 16 * 2, kUmmaB3 = kUmmaB2 + 32 * 32 * 2, kUmmaBBytes = kUmmaB3 + 16 * 32 * 2;

__host__ inline void mlp_pack_umma(const float* P, uint16_t* img /*[kUmmaBBytes / 2]*/) {
  std::memset(img, 0, kUmmaBBytes);
  for (int n = 0; n < kMlpHidden; ++n)
    for (int k = 0; k < kMlpIn; ++k) img[(kUmmaB1 + umma_off(n, k, 16)) / 2] = bf16_bits_rn(P[kMlpW1 + n * kMlpIn + k]);
  for (int n = 0; n < kMlpHidden; ++n)
    for (int k = 0; k < kMlpHidden; ++k)
      img[(kUmmaB2 + umma_off(n, k, 32)) / 2] = bf16_bits_rn(P[kMlpW2 + n * kMlpHidden + k]);
  for (int k = 0; k < kMlpHidden; ++k) img[(kUmmaB3 + umma_off(0, k, 32)) / 2] = bf16_bits_rn(P[kMlpW3 + k]);
}

#ifdef __CUDACC__
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_dst), "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (TMEM) = A B^T (+ D when accumulate), one CTA, kind::f16.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrives on the mbarrier once every earlier tcgen05 operation of this thread is done.
__device__ __forceinline__ void umma_commit(uint32_t mbar_smem) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_smem)
               : "memory");
}
// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  return __uint_as_float(r);
}

__device__ __forceinline__ void umma_mbar_init(uint32_t mbar_smem) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_smem) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool umma_mbar_wait(uint32_t mbar_smem, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar_smem), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// GELU(d + b) of 32 columns (packed BF16 pairs), stored into row r of a K = 32 operand.
__device__ __forceinline__ void umma_store_hidden(uint8_t* A, int r, const float (&d)[32], const float* b) {
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    uint4 w;
    w.x = gelu_bf16x2(d[8 * g + 0] + b[8 * g + 0], d[8 * g + 1] + b[8 * g + 1]);
    w.y = gelu_bf16x2(d[8 * g + 2] + b[8 * g + 2], d[8 * g + 3] + b[8 * g + 3]);
    w.z = gelu_bf16x2(d[8 * g + 4] + b[8 * g + 4], d[8 * g + 5] + b[8 * g + 5]);
    w.w = gelu_bf16x2(d[8 * g + 6] + b[8 * g + 6], d[8 * g + 7] + b[8 * g + 7]);
    *reinterpret_cast<uint4*>(A + umma_off(r, 8 * g, 32)) = w;
  }
}

// ---- the closure inside the step kernel: 128-cell groups of four consumer warps -----
// The step kernel's 8 consumer warps form two groups of four (warps 0-3 and 4-7); warp
// w owns TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31, so the four warps of a group together
// hold the 128 rows of one M = 128 tile: a group evaluates the network for its 128 cells
// (one 32-cell segment per warp) with three tcgen05.mma layers issued by one thread.
// Each group owns 64 TMEM columns (D1 and D3 at +0, D2 at +32; 128 per CTA), its A
// operands and an mbarrier; the weight image is shared.  The four warps meet at a named
// barrier before every layer; the barrier also reduces a failure flag (a timed-out
// completion wait, or a ring wait that ran out before the segment), so that the warps of
// a group always leave together and no barrier can wait for a warp that has left.
constexpr int kStepUmmaGroups = 2;
constexpr uint32_t kStepUmmaTmemCols = 128;  // power of two >= 32, per CTA
constexpr size_t kStepUmmaA1 = 128 * 16 * 2, kStepUmmaA2 = 128 * 32 * 2;
// shared memory of the tcgen05 closure: alignment slack, the weight image, the A
// operands of each group, an mbarrier per group and the TMEM address slot
constexpr size_t kStepUmmaBytes =
    128 + kUmmaBBytes + kStepUmmaGroups * (kStepUmmaA1 + kStepUmmaA2) + 8 * kStepUmmaGroups + 8;

struct UmmaGroup {
  uint8_t* a1;  // 128 x 16 BF16 (inputs, K padded with zeros)
  uint8_t* a2;  // 128 x 32 BF16 (hidden activations)
  uint64_t dA1, dA2lo, dA2hi, dB1, dB2lo, dB2hi, dB3lo, dB3hi;  // operand descriptors
  uint32_t mbar;       // shared address of the group's completion mbarrier
  uint32_t tmem;       // the group's TMEM columns, lane 0
  uint32_t lane_addr;  // the same, at this warp's 32 lanes
  uint32_t phase;      // parity of the next completion
  int issued;          // commits issued (issuing thread)
  int row;             // this thread's cell = row of the tile
  int bar_id;          // named barrier of the group (1 + group)
  int limit;           // polls of a completion wait
  bool issuer, failed;
};

// OR of v over the 128 threads of a group, at its named barrier.
__device__ __forceinline__ bool group_any(int bar_id, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "barrier.cta.red.or.pred p, %2, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(bar_id)
      : "memory");
  return r != 0;
}

// nu_t / nu_0 of this thread's cell; all 128 threads of the group call it together.
// Returns NaN when the group has failed (the caller then keeps the Smagorinsky tau and
// leaves the item loop at its next group agreement).
__device__ __forceinline__ float mlp_nut_umma(const float (&x)[kMlpIn], UmmaGroup& g, const float* bias) {
  *reinterpret_cast<uint4*>(g.a1 + umma_off(g.row, 0, 16)) =
      make_uint4(bf16x2_of(x[0], x[1]), bf16x2_of(x[2], x[3]), bf16x2_of(x[4], x[5]), bf16x2_of(x[6], x[7]));
  constexpr uint32_t id32 = umma_idesc_bf16(kUmmaRows, 32), id16 = umma_idesc_bf16(kUmmaRows, 16);
  bool ok = true;
  float d[32];
#pragma unroll 1
  for (int layer = 0; layer < 3; ++layer) {
    fence_async_smem();  // this thread's operand writes, visible to the tensor cores
    tc_fence_before();
    if (group_any(g.bar_id, g.failed || !ok)) {
      g.failed = true;
      return __int_as_float(0x7fc00000);
    }
    tc_fence_after();
    if (g.issuer) {
      if (layer == 0) {
        umma_bf16(g.tmem, g.dA1, g.dB1, id32, 0u);
      } else if (layer == 1) {
        umma_bf16(g.tmem + 32, g.dA2lo, g.dB2lo, id32, 0u);
        umma_bf16(g.tmem + 32, g.dA2hi, g.dB2hi, id32, 1u);
      } else {
        umma_bf16(g.tmem, g.dA2lo, g.dB3lo, id16, 0u);
        umma_bf16(g.tmem, g.dA2hi, g.dB3hi, id16, 1u);
      }
      umma_commit(g.mbar);
      ++g.issued;
    }
    // tcgen05.ld is warp-collective: a warp reads only when all its lanes saw the phase
    ok = __all_sync(0xffffffffu, umma_mbar_wait(g.mbar, g.phase, g.limit));
    g.phase ^= 1u;
    if (ok) {
      tc_fence_after();
      if (layer < 2) {
        tmem_ld32(g.lane_addr + (layer == 0 ? 0u : 32u), d);
        umma_store_hidden(g.a2, g.row, d, bias + 32 * layer);
      }
    }
  }
  g.failed = g.failed || !ok;  // agreed on at the group's next barrier
  if (!ok) return __int_as_float(0x7fc00000);
  const float o = tmem_ld1(g.lane_addr) + bias[64];
  tc_fence_before();
  return softplus_f(o);
}
#endif

}  // namespace aerosim
