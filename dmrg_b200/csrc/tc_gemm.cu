// Split-precision grouped GEMM, warp-specialized: TMA -> tcgen05.mma (TMEM) -> epilogue.
//
// Each FP64 operand x is carried as a pair (hi, lo) of low-precision numbers,
// hi = rn(x), lo = rn(x - hi), and every product a.b is evaluated as
//     a_hi.b_hi + a_hi.b_lo + a_lo.b_hi          (the lo.lo term is dropped)
// by three tcgen05.mma instructions accumulating into one FP32 TMEM accumulator.
// Element types: BF16 pairs (kind::f16, K=16 per instruction) or TF32 pairs in
// 32-bit containers (kind::tf32, K=8 per instruction).
//
// Operand blocks are row-major with K contiguous in the pair layout of split.h:
// each 128-byte chunk of a row holds 64 bytes of hi parts and the 64 bytes of
// their lo parts.  One 2-D tensor map per block with 128-byte swizzle brings a
// k-tile (one chunk per row, both halves) in one TMA instruction of 128-byte
// rows, straight into the UMMA canonical K-major SW128 layout (8-row atoms of
// 1 KB); the hi k-steps sit at byte 0 and 32 of each row, the lo k-steps at 64
// and 96.  Rows past the block edge are zero-filled by TMA.
//
// Roles (192 threads):
//   warp 0      TMA producer: walks the work unit's k-tiles over its segments,
//               fills a STAGES-deep smem ring (full/empty mbarrier pairs)
//   warp 1      TMEM allocator and MMA issuer: 3 products x k-steps per k-tile,
//               commits each k-tile to its ring slot's empty barrier and the
//               last one of a unit to the accumulator's full barrier
//   warps 2..5  epilogue: tcgen05.ld of the 128 accumulator rows (warp w reads
//               TMEM lanes 32*(w%4)..), writes the unit's result
// Two TMEM accumulators (2 x 256 columns) let the epilogue of one unit overlap
// the MMAs of the next.
//
// Work unit = (output tile of 128 rows x <=256 columns, a range of its k-tiles).
// Long tiles are split along K so every SM gets work; a split unit writes its
// FP32 partial to a workspace slot and split_reduce sums the slots in a fixed
// order (deterministic).  The MMA N of a unit is its tile's column count
// rounded up to 16, chosen at run time in the instruction descriptor.
//
// Every wait is bounded: a timed-out wait sets the error word, the thread stops
// its role, the CTA drains and frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "split.h"

namespace dmrgx {

namespace {

constexpr int THREADS = 192;
constexpr int TM = 128;
constexpr int TNMAX = 256;                    // widest tile; also the workspace row stride
constexpr int ROWB = 128;                     // bytes per row of one k-tile (hi + lo)
constexpr int HALF = 64;                      // byte offset of the lo parts in a row
constexpr int A_BYTES = TM * ROWB;            // 16 KB
constexpr int SBO = 8 * ROWB;                 // 1 KB between 8-row atoms
constexpr uint64_t WAIT_NS = 2000000000ull;  // a wait gives up after 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// try_wait suspends in hardware until the phase completes or a short time
// limit passes; the loop gives up after WAIT_NS of wall time.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (!mbar_try(bar, parity))
    if (globaltimer_ns() - t0 > WAIT_NS) return false;
  return true;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// bring a tensor map (global memory) into the TMA descriptor cache
__device__ __forceinline__ void prefetch_map(const CUtensorMap* m) {
  asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(m)) : "memory");
}
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  // K-major, 128-byte swizzle: LBO unused (1), SBO = 1 KB, version 1, layout 2
  return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(SBO >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}
template <int EB>
__device__ __forceinline__ uint32_t instr_desc(int n) {
  constexpr uint32_t fmt = EB == 2 ? 1u : 2u;  // BF16 (kind::f16) or TF32 (kind::tf32)
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(TM >> 4) << 24);
}
template <int EB>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accum) {
  if (EB == 2)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
template <int EB>
__device__ __forceinline__ void split_f32(float v, uint32_t& hi, uint32_t& lo) {
  if (EB == 2) {
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
  } else {
    hi = tf32_rna(v);
    lo = tf32_rna(v - __uint_as_float(hi));
  }
}

// (hi, lo) pairs of EPC = 16 / EB consecutive values (16 bytes of each half)
// at logical k of a pair-layout row; a group never crosses a chunk (k is a
// multiple of EPC)
template <int EB>
__device__ __forceinline__ void put_group(uint8_t* c_pair, int64_t rbase, int64_t k,
                                          const float* v) {
  constexpr int CH = 64 / EB;
  uint32_t hw[4], lw[4];
  if (EB == 2) {
#pragma unroll
    for (int p = 0; p < 4; p++) {
      uint32_t h0, l0, h1, l1;
      split_f32<2>(v[2 * p], h0, l0);
      split_f32<2>(v[2 * p + 1], h1, l1);
      hw[p] = h0 | (h1 << 16);
      lw[p] = l0 | (l1 << 16);
    }
  } else {
#pragma unroll
    for (int p = 0; p < 4; p++) split_f32<4>(v[p], hw[p], lw[p]);
  }
  const int64_t eoff = (rbase + pair_off(k, CH)) * EB;
  *reinterpret_cast<uint4*>(c_pair + eoff) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4*>(c_pair + eoff + HALF) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// Final store of 16 consecutive columns of one row (cols [col0, col0+16)).
// Stage 1 (OUT_SPLIT): (hi, lo) pairs in pair layout, groups of 16 / EB columns
// (n1p and col0 are multiples of a group).  Complex data: columns are (Re, Im)
// pairs and the row is written in the expanded form of split.h, rows 2q, 2q+1.
template <int EB, bool OUT_SPLIT>
__device__ __forceinline__ void store16(const SOut& o, int row, int col0, const float* v,
                                        uint8_t* c_pair, double* c64) {
  if (OUT_SPLIT) {
    constexpr int EPC = 16 / EB;
    const int64_t q = row / o.grp;
    const int64_t kb = (int64_t)(row % o.grp) * o.ldc;
    if (!o.cplx) {
      const int64_t rbase = o.c_off + q * o.rstride;
#pragma unroll
      for (int gq = 0; gq < 16 / EPC; gq++) {
        if (col0 + gq * EPC >= o.ldc) break;
        put_group<EB>(c_pair, rbase, kb + col0 + gq * EPC, v + gq * EPC);
      }
    } else {
      const int64_t r0 = o.c_off + 2 * q * o.rstride, r1 = r0 + o.rstride;
      float va[16], vb[16];
#pragma unroll
      for (int t = 0; t < 8; t++) {
        va[2 * t] = v[2 * t];
        va[2 * t + 1] = -v[2 * t + 1];
        vb[2 * t] = v[2 * t + 1];
        vb[2 * t + 1] = v[2 * t];
      }
#pragma unroll
      for (int gq = 0; gq < 16 / EPC; gq++) {
        if (col0 + gq * EPC >= o.ldc) break;
        put_group<EB>(c_pair, r0, kb + col0 + gq * EPC, va + gq * EPC);
        put_group<EB>(c_pair, r1, kb + col0 + gq * EPC, vb + gq * EPC);
      }
    }
  } else {
    const int64_t rbase = o.c_off + (int64_t)row * o.ldc + col0;
#pragma unroll
    for (int i = 0; i < 16; i++)
      if (col0 + i < o.n) c64[rbase + i] = (double)v[i];
  }
}

// TNX: widest tile (MMA N) of this instantiation; STAGES: depth of the ring.
// Configurations: (256, 4) and (128, 7) with one CTA per SM -- the narrow one
// keeps more k-tiles in flight for the same shared memory -- and (128, 3),
// (64, 4) sized for two CTAs per SM (one waits on TMA while the other computes;
// the two accumulator pairs use all 512 TMEM columns).
template <int EB, bool OUT_SPLIT, int TNX, int STAGES>
__global__ void __launch_bounds__(THREADS, 2)
tc_grouped_gemm(const CUtensorMap* __restrict__ maps, const SUnit* __restrict__ units,
                const int* __restrict__ cta_begin, const SOut* __restrict__ outs,
                const SSeg2* __restrict__ segs, uint8_t* __restrict__ c_pair,
                double* __restrict__ c64, float* __restrict__ ws, int* __restrict__ err) {
  constexpr int B_BYTES = TNX * ROWB;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = 2 * TNX;  // two accumulators
  extern __shared__ uint8_t smem_raw[];
  // 1024-aligned ring (the swizzle pattern repeats every 512 B)
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);

  constexpr int BK = HALF / EB;   // elements (of each half) per k-tile
  constexpr int NKS = BK / (32 / EB);  // MMA k-steps (32 bytes each) per k-tile
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t sbase = smem_u32(smem);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(smem_u32(&tfull[a]), 1);
      mbar_init(smem_u32(&tempty[a]), 4);  // one arrive per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  // programmatic dependent launch: the set-up above may overlap the previous
  // kernel's tail; operands and outputs are touched only after it completed
  // the tensor maps of this CTA's units go to the descriptor cache while the
  // previous kernel finishes: maps, units and segments are plan data, written
  // before any kernel of the matvec (operands are read only after pdl_wait)
  if (warp == 0) {
    const int ub = cta_begin[blockIdx.x], ue = cta_begin[blockIdx.x + 1];
    for (int u = ub; u < ue; u++) {
      const SOut o = outs[units[u].out];
      for (int q = lane; q < o.seg_count; q += 32) {
        const SSeg2 sg = segs[o.seg_begin + q];
        prefetch_map(maps + sg.amap);
        prefetch_map(maps + sg.bmap);
      }
    }
  }
  pdl_wait();
  pdl_launch_dependents();
  const uint32_t tmem = *tmem_slot;
  const int ubeg = cta_begin[blockIdx.x], uend = cta_begin[blockIdx.x + 1];

  if (warp == 0) {
    // ------------------------------------------------------------ TMA producer
    if (lane == 0) {
      uint32_t g = 0;
      bool ok = true;
      for (int u = ubeg; u < uend && ok; u++) {
        const SUnit un = units[u];
        const SOut o = outs[un.out];
        // locate the unit's first k-tile
        int s = o.seg_begin, base = 0;
        while (s < o.seg_begin + o.seg_count && base + segs[s].nkt <= un.kt0) {
          base += segs[s].nkt;
          s++;
        }
        int kin = un.kt0 - base;
        for (int kt = un.kt0; kt < un.kt1; kt++) {
          const SSeg2 sg = segs[s];
          const uint32_t slot = g % STAGES;
          if (g >= STAGES) ok = mbar_wait(smem_u32(&empty[slot]), ((g / STAGES) - 1) & 1);
          if (!ok) {
            atomicExch(err, 2);
            break;
          }
          const uint32_t st = sbase + slot * STAGE_BYTES;
          const uint32_t bar = smem_u32(&full[slot]);
          mbar_expect_tx(bar, (uint32_t)(A_BYTES + sg.brows * ROWB));
          tma_load_2d(st, maps + sg.amap, kin * 2 * BK, un.tm * TM, bar);
          tma_load_2d(st + A_BYTES, maps + sg.bmap, kin * 2 * BK, un.tn * o.tnw, bar);
          g++;
          if (++kin >= sg.nkt) {
            kin = 0;
            s++;
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t g = 0, ua = 0;
      bool ok = true;
      for (int u = ubeg; u < uend && ok; u++) {
        const SUnit un = units[u];
        if (un.kt1 <= un.kt0) continue;
        const SOut o = outs[un.out];
        const int ncols = min(o.tnw, o.n - un.tn * o.tnw);
        const int nmma = (ncols + 15) & ~15;
        const uint32_t idesc = instr_desc<EB>(nmma);
        const uint32_t acc = ua & 1;
        if (ua >= 2) ok = mbar_wait(smem_u32(&tempty[acc]), ((ua / 2) - 1) & 1);
        if (!ok) {
          atomicExch(err, 3);
          break;
        }
        tc_fence_after();
        const uint32_t tacc = tmem + acc * TNX;
        int s = o.seg_begin, base = 0;
        while (s < o.seg_begin + o.seg_count && base + segs[s].nkt <= un.kt0) {
          base += segs[s].nkt;
          s++;
        }
        int kin = un.kt0 - base;
        for (int kt = un.kt0; kt < un.kt1; kt++) {
          const SSeg2 sg = segs[s];
          const uint32_t slot = g % STAGES;
          ok = mbar_wait(smem_u32(&full[slot]), (g / STAGES) & 1);
          if (!ok) {
            atomicExch(err, 4);
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + slot * STAGE_BYTES;
          const uint32_t a_t = st, b_t = st + A_BYTES;
#pragma unroll
          for (int j = 0; j < NKS; j++) {
            const uint32_t ko = j * 32;
            const uint64_t ah = sw128_desc(a_t + ko), al = sw128_desc(a_t + HALF + ko);
            const uint64_t bh = sw128_desc(b_t + ko), bl = sw128_desc(b_t + HALF + ko);
            mma<EB>(tacc, ah, bh, idesc, (kt > un.kt0 || j > 0) ? 1u : 0u);
            mma<EB>(tacc, ah, bl, idesc, 1u);
            mma<EB>(tacc, al, bh, idesc, 1u);
          }
          mma_commit(smem_u32(&empty[slot]));
          g++;
          if (++kin >= sg.nkt) {
            kin = 0;
            s++;
          }
        }
        if (!ok) break;
        mma_commit(smem_u32(&tfull[acc]));
        ua++;
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue (warps 2..5)
    const int q = warp & 3;              // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    uint32_t ua = 0;
    bool ok = true;
    for (int u = ubeg; u < uend && ok; u++) {
      const SUnit un = units[u];
      const SOut o = outs[un.out];
      const int ncols = min(o.tnw, o.n - un.tn * o.tnw);
      const int nmma = (ncols + 15) & ~15;
      const int m0 = un.tm * TM, n0 = un.tn * o.tnw;
      const bool has = un.kt1 > un.kt0;
      const uint32_t acc = ua & 1;
      if (has) {
        ok = mbar_wait(smem_u32(&tfull[acc]), (ua / 2) & 1);
        if (!ok) {
          atomicExch(err, 5);
          break;
        }
        tc_fence_after();
      }
      const uint32_t taddr = tmem + acc * TNX + ((uint32_t)(q * 32) << 16);
      for (int cc = 0; cc < nmma; cc += 16) {
        float v[16];
        if (has) {
          tmem_ld16(taddr + cc, v);
        } else {
#pragma unroll
          for (int i = 0; i < 16; i++) v[i] = 0.f;
        }
        if (m0 + row >= o.m) continue;
        if (un.slot >= 0) {
          float* p = ws + ((int64_t)un.slot * TM + row) * TNMAX + cc;
#pragma unroll
          for (int i = 0; i < 16; i += 4)
            *reinterpret_cast<float4*>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        } else {
          store16<EB, OUT_SPLIT>(o, m0 + row, n0 + cc, v, c_pair, c64);
        }
      }
      if (has) {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&tempty[acc]));
        ua++;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
}

// 4 values as (hi, lo) pairs at logical k of a pair-layout row
template <int EB>
__device__ __forceinline__ void put4(uint8_t* c_pair, int64_t rbase, int64_t k, float4 v) {
  constexpr int CH = 64 / EB;
  const int64_t e = rbase + pair_off(k, CH);
  uint32_t h[4], l[4];
  split_f32<EB>(v.x, h[0], l[0]);
  split_f32<EB>(v.y, h[1], l[1]);
  split_f32<EB>(v.z, h[2], l[2]);
  split_f32<EB>(v.w, h[3], l[3]);
  if (EB == 2) {
    *reinterpret_cast<uint2*>(c_pair + e * 2) = make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
    *reinterpret_cast<uint2*>(c_pair + e * 2 + HALF) = make_uint2(l[0] | (l[1] << 16), l[2] | (l[3] << 16));
  } else {
    *reinterpret_cast<uint4*>(c_pair + e * 4) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(c_pair + e * 4 + HALF) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// Final store of 4 consecutive columns of one row (cols [col0, col0+4)).
template <int EB, bool OUT_SPLIT>
__device__ __forceinline__ void store4(const SOut& o, int row, int col0, float4 v,
                                       uint8_t* c_pair, double* c64) {
  if (OUT_SPLIT) {
    if (col0 >= o.ldc) return;  // ldc is a multiple of 4 elements
    const int64_t q = row / o.grp;
    const int64_t k = (int64_t)(row % o.grp) * o.ldc + col0;
    if (!o.cplx) {
      put4<EB>(c_pair, o.c_off + q * o.rstride, k, v);
    } else {
      const int64_t r0 = o.c_off + 2 * q * o.rstride;
      put4<EB>(c_pair, r0, k, make_float4(v.x, -v.y, v.z, -v.w));
      put4<EB>(c_pair, r0 + o.rstride, k, make_float4(v.y, v.x, v.w, v.z));
    }
  } else {
    const int64_t e = o.c_off + (int64_t)row * o.ldc + col0;
    if (col0 < o.n) c64[e] = (double)v.x;
    if (col0 + 1 < o.n) c64[e + 1] = (double)v.y;
    if (col0 + 2 < o.n) c64[e + 2] = (double)v.z;
    if (col0 + 3 < o.n) c64[e + 3] = (double)v.w;
  }
}

constexpr int RED_ROWS = 4;  // rows of one K-split tile per reduction block

// Sum the K-split partials of a tile in slot order (deterministic) and store
// them; one thread per (row, 4 columns), 4 rows per block.
template <int EB, bool OUT_SPLIT>
__global__ void __launch_bounds__(256)
split_reduce(const SRed* __restrict__ reds, const SRedBlk* __restrict__ blks,
             const SOut* __restrict__ outs, const float* __restrict__ ws,
             uint8_t* __restrict__ c_pair, double* __restrict__ c64) {
  pdl_wait();
  pdl_launch_dependents();
  const SRedBlk b = blks[blockIdx.x];
  const SRed rd = reds[b.red];
  const SOut o = outs[rd.out];
  const int m0 = rd.tm * TM, n0 = rd.tn * o.tnw;
  const int rows = min(TM, o.m - m0);
  const int ncols = min(o.tnw, o.n - n0);
  const int g4 = ((ncols + 15) & ~15) / 4;  // float4 groups per row
  const int r = b.r0 + threadIdx.x / 64, g = threadIdx.x % 64;
  if (r >= rows || r >= b.r0 + RED_ROWS || g >= g4) return;
  const float* p = ws + ((int64_t)rd.slot0 * TM + r) * TNMAX + g * 4;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int s = 0; s < rd.nslots; s++) {
    const float4 t = *reinterpret_cast<const float4*>(p + (int64_t)s * TM * TNMAX);
    acc.x += t.x;
    acc.y += t.y;
    acc.z += t.z;
    acc.w += t.w;
  }
  store4<EB, OUT_SPLIT>(o, m0 + r, n0 + g * 4, acc, c_pair, c64);
}

}  // namespace

int tc_configs() { return 4; }
int tc_cfg_tn(int cfg) { return cfg == 0 ? 256 : cfg == 3 ? 64 : 128; }
int tc_cfg_stages(int cfg) { return cfg == 0 ? 4 : cfg == 1 ? 7 : cfg == 2 ? 3 : 4; }
int tc_cfg_ctas_per_sm(int cfg) { return cfg >= 2 ? 2 : 1; }
int tc_smem_bytes(int cfg) {
  const int st = tc_cfg_stages(cfg);
  return st * (A_BYTES + tc_cfg_tn(cfg) * ROWB) + 1024 + (2 * st + 4) * 8 + 16;
}
int tc_tile_m() { return TM; }
int tc_tile_n() { return TNMAX; }  // workspace row stride (floats)
int tc_ktile_bytes() { return ROWB; }

// Opt the kernels into their shared memory on the current device (once per plan,
// outside any stream capture).
cudaError_t prepare_tc_gemm() {
  cudaError_t e = cudaSuccess;
#define DMRGX_TC_ATTR(EB, OS, TN, ST, CFG)                                    \
  if (e == cudaSuccess)                                                       \
    e = cudaFuncSetAttribute(tc_grouped_gemm<EB, OS, TN, ST>,                 \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes(CFG));
  DMRGX_TC_ATTR(2, true, 256, 4, 0)
  DMRGX_TC_ATTR(2, false, 256, 4, 0)
  DMRGX_TC_ATTR(4, true, 256, 4, 0)
  DMRGX_TC_ATTR(4, false, 256, 4, 0)
  DMRGX_TC_ATTR(2, true, 128, 7, 1)
  DMRGX_TC_ATTR(2, false, 128, 7, 1)
  DMRGX_TC_ATTR(4, true, 128, 7, 1)
  DMRGX_TC_ATTR(4, false, 128, 7, 1)
  DMRGX_TC_ATTR(2, true, 128, 3, 2)
  DMRGX_TC_ATTR(2, false, 128, 3, 2)
  DMRGX_TC_ATTR(4, true, 128, 3, 2)
  DMRGX_TC_ATTR(4, false, 128, 3, 2)
  DMRGX_TC_ATTR(2, true, 64, 4, 3)
  DMRGX_TC_ATTR(2, false, 64, 4, 3)
  DMRGX_TC_ATTR(4, true, 64, 4, 3)
  DMRGX_TC_ATTR(4, false, 64, 4, 3)
#undef DMRGX_TC_ATTR
  return e;
}

cudaError_t launch_tc_gemm(int eb, bool out_split, int cfg, const CUtensorMap* maps,
                           const SUnit* units, const int* cta_begin, int nctas, const SOut* outs,
                           const SSeg2* segs, void* c_pair, double* c64, float* ws,
                           const SRed* reds, const SRedBlk* redblk, int nredblk, int* err,
                           cudaStream_t st) {
  if (nctas <= 0) return cudaSuccess;
  const int sm = tc_smem_bytes(cfg);
#define DMRGX_TC_LAUNCH(EB, OS, TN, STG)                                                      \
  do {                                                                                        \
    cudaError_t e_ = launch_pdl(tc_grouped_gemm<EB, OS, TN, STG>, nctas, THREADS, sm, st,      \
                                maps, units, cta_begin, outs, segs, (uint8_t*)c_pair, c64, ws, \
                                err);                                                         \
    if (e_ == cudaSuccess && nredblk > 0)                                                     \
      e_ = launch_pdl(split_reduce<EB, OS>, nredblk, 256, 0, st, reds, redblk, outs,          \
                      (const float*)ws, (uint8_t*)c_pair, c64);                               \
    if (e_ != cudaSuccess) return e_;                                                         \
  } while (0)
  if (cfg == 0) {
    if (eb == 2) {
      if (out_split) DMRGX_TC_LAUNCH(2, true, 256, 4);
      else DMRGX_TC_LAUNCH(2, false, 256, 4);
    } else {
      if (out_split) DMRGX_TC_LAUNCH(4, true, 256, 4);
      else DMRGX_TC_LAUNCH(4, false, 256, 4);
    }
  } else if (cfg == 1) {
    if (eb == 2) {
      if (out_split) DMRGX_TC_LAUNCH(2, true, 128, 7);
      else DMRGX_TC_LAUNCH(2, false, 128, 7);
    } else {
      if (out_split) DMRGX_TC_LAUNCH(4, true, 128, 7);
      else DMRGX_TC_LAUNCH(4, false, 128, 7);
    }
  } else if (cfg == 2) {
    if (eb == 2) {
      if (out_split) DMRGX_TC_LAUNCH(2, true, 128, 3);
      else DMRGX_TC_LAUNCH(2, false, 128, 3);
    } else {
      if (out_split) DMRGX_TC_LAUNCH(4, true, 128, 3);
      else DMRGX_TC_LAUNCH(4, false, 128, 3);
    }
  } else {
    if (eb == 2) {
      if (out_split) DMRGX_TC_LAUNCH(2, true, 64, 4);
      else DMRGX_TC_LAUNCH(2, false, 64, 4);
    } else {
      if (out_split) DMRGX_TC_LAUNCH(4, true, 64, 4);
      else DMRGX_TC_LAUNCH(4, false, 64, 4);
    }
  }
#undef DMRGX_TC_LAUNCH
  return cudaGetLastError();
}

}  // namespace dmrgx
