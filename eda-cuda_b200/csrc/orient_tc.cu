// SPDX-License-Identifier: Apache-2.0
// The float32 axis transforms of the orientation on the 5th-generation tensor cores (sm_100a):
// out = A B^T per element rows, A the field's rows along its contiguous axis (K = that axis),
// B the n x n basis (forward DCT-II, inverse cosine or inverse sine) of that axis.
//
// Precision: split products with float32 accumulation in tensor memory, the float32 operand x split
// into hi + lo and the product taken as hi_a hi_b + hi_a lo_b + lo_a hi_b (three MMAs; the dropped
// lo_a lo_b term is below 2^-2p of the product). 3xTF32 (kind::tf32): hi = tf32(x), lo =
// tf32(x - hi), about 22 bits of every operand; BF16x3 (kind::f16 on bfloat16): hi = bf16(x), lo =
// bf16(x - hi), about 16 bits, at twice the MMA rate. (The reference runs these transforms with
// cuFFT in float32, cpp/src/method/orientation.cu:674-767 of eda-cuda.) The basis is split once on
// the host; the field tile is split in shared memory after its TMA load.
//
// Kernel (one 128 x 128 output tile per CTA, 192 threads):
//   warp 4      TMA producer: A tile (128 rows x 32 floats, 128B swizzle) and the hi and lo basis
//               tiles per k-block into a 3-stage ring (full / empty mbarriers);
//   warps 0-3   split the A tile into hi and lo tiles (3xTF32: hi in place, 128B swizzle; BF16x3:
//               two bfloat16 tiles of 64-byte rows in the 64B swizzle), fence the async proxy,
//               arrive on the stage's split barrier; then the epilogue: tcgen05.ld of their TMEM
//               lane quarter and the transposed store;
//   warp 5      allocates 128 TMEM columns; one thread issues the split MMAs of every k-block
//               (3 x 4 kind::tf32 with K = 8, or 3 x 2 kind::f16 with K = 16; M = N = 128) and
//               commits each stage back to the producer.
// The store writes the tile transposed: the transformed axis becomes the slowest axis of the
// element and the next axis the contiguous one (a rotation of the layout), so every transform of
// the orientation reads K-major rows, and D passes bring a field back to its layout.
// Every wait is bounded (about 2 s): on expiry the kernel sets *err, waits (bounded) for its own
// TMA copies, frees its tensor memory and returns.
#include "orient.cuh"

#include <cuda.h>

#include <cstring>
#include <mutex>

namespace edab {
namespace tc {

constexpr int kBM = 128, kBN = 128, kBK = 32, kStages = 3;
constexpr int kThreadsTc = 192;
constexpr unsigned long long kWaitNs = 2000000000ull;

// The stage layout of a split mode. 3xTF32: [A hi (TMA, then split in place) | A lo | B hi | B lo],
// 16 KiB each, rows of 128 bytes. BF16x3: [A float32 (TMA) 16 KiB | A hi | A lo | B hi | B lo], the
// bfloat16 tiles 8 KiB each, rows of 64 bytes. Every tile starts on a 1024-byte boundary.
template <bool BF16>
struct Stage {
  static constexpr int kTileF32 = kBM * kBK * 4;                      // 16 KiB: the float32 A tile
  static constexpr int kTileOp = BF16 ? kBM * kBK * 2 : kBM * kBK * 4;  // one operand tile
  static constexpr int kAhi = BF16 ? kTileF32 : 0;
  static constexpr int kAlo = kAhi + kTileOp;
  static constexpr int kBhi = kAlo + kTileOp;
  static constexpr int kBlo = kBhi + kTileOp;
  static constexpr int kBytes = kBlo + kTileOp;
  static constexpr int kTmaBytes = kTileF32 + 2 * kTileOp;  // A float32, B hi, B lo
  static constexpr int kSmem = kStages * kBytes + 1024 + 256;
};

// Instruction descriptors (D float32, both operands K-major, N, M): kind::tf32 with tf32 A and B;
// kind::f16 with bfloat16 A and B.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(kBN >> 3) << 17) |
                                (static_cast<uint32_t>(kBM >> 4) << 24);
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kBN >> 3) << 17) |
                                (static_cast<uint32_t>(kBM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Shared-memory matrix descriptor of a K-major tile with the 128-byte swizzle: rows of 128 bytes,
// 8-row groups 1024 bytes apart (SBO), version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3fffu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(1024 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(2) << 61);
}
// The same for a K-major tile with the 64-byte swizzle: rows of 64 bytes, 8-row groups 512 bytes
// apart, layout SWIZZLE_64B.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3fffu) | (static_cast<uint64_t>(1) << 16) |
         (static_cast<uint64_t>(512 >> 4) << 32) | (static_cast<uint64_t>(1) << 46) |
         (static_cast<uint64_t>(4) << 61);
}
__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete; false after about kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = now_ns();
  while (!mbar_try(bar, parity)) {
    if (now_ns() - t0 > kWaitNs) return false;
  }
  return true;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int32_t x, int32_t y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdescTf32), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdescBf16), "r"(accumulate)
      : "memory");
}
// bfloat16 of x rounded to nearest even, as raw bits (x finite or infinite; NaN stays NaN).
__device__ __forceinline__ uint32_t bf16_bits(float x) {
  uint32_t r;
  asm("{\n\t.reg .b16 h;\n\tcvt.rn.bf16.f32 h, %1;\n\tmov.b32 %0, {h, h};\n\t}" : "=r"(r) : "f"(x));
  return r & 0xffffu;
}
__device__ __forceinline__ float bf16_value(uint32_t bits) { return __uint_as_float(bits << 16); }
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Row m of the pass (element b = m / rows, row r = m % rows = hi * n_lo + lo) stores its column j
// at b * f_out + j * s_j + hi * pitch_out + lo.
struct RotOut {
  int64_t M;          // rows of the batch (B * rows)
  int32_t N;          // output columns (the transformed axis)
  int32_t kblocks;    // ceil(K / 32)
  int32_t npad;       // row offset of the lo basis in the basis tensor
  int64_t rows;       // rows per element
  int64_t n_lo;       // extent of the fastest row axis
  int64_t pitch_out;  // padded extent of the output's contiguous axis
  int64_t s_j;        // output stride of the transformed axis
  int64_t f_out;      // output samples per element
};

template <bool BF16>
__global__ void __launch_bounds__(kThreadsTc, 1)
    gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, RotOut ro,
            float* __restrict__ out, const int32_t* __restrict__ run, int32_t* __restrict__ err) {
  using L = Stage<BF16>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStages * L::kBytes);
  // bars: full[kStages], split[kStages], empty[kStages], acc
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * kStages + 1);
  __shared__ int32_t active_s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * kBM;
  const int32_t n0 = static_cast<int32_t>(blockIdx.x) * kBN;
  if (threadIdx.x == 0) {
    // a tile whose rows all belong to elements that do not run is skipped
    const int64_t m1 = min(m0 + kBM, ro.M) - 1;
    int32_t act = 0;
    for (int64_t b = m0 / ro.rows; b <= m1 / ro.rows; ++b) act |= run[b] != 0;
    active_s = act;
    if (act) {
      for (int s = 0; s < kStages; ++s) {
        mbar_init(smem_u32(&bars[s]), 1);
        mbar_init(smem_u32(&bars[kStages + s]), 128);
        mbar_init(smem_u32(&bars[2 * kStages + s]), 1);
      }
      mbar_init(smem_u32(&bars[3 * kStages]), 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  if (!active_s) return;
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  bool ok = true;
  if (warp == 4) {
    if (lane == 0) {
      int32_t issued = 0;
      for (int32_t kb = 0; kb < ro.kblocks; ++kb) {
        const int s = kb % kStages;
        const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
        if (!mbar_wait(smem_u32(&bars[2 * kStages + s]), ph ^ 1u)) {
          ok = false;
          break;
        }
        unsigned char* st = base + s * L::kBytes;
        const uint32_t full = smem_u32(&bars[s]);
        mbar_expect_tx(full, L::kTmaBytes);
        tma_load_2d(smem_u32(st), &ta, kb * kBK, static_cast<int32_t>(m0), full);
        tma_load_2d(smem_u32(st + L::kBhi), &tb, kb * kBK, n0, full);
        tma_load_2d(smem_u32(st + L::kBlo), &tb, kb * kBK, ro.npad + n0, full);
        issued = kb + 1;
      }
      // the copies of the last stages complete before the CTA may leave
      for (int32_t kb = max(0, issued - kStages); kb < issued; ++kb) {
        if (!mbar_wait(smem_u32(&bars[kb % kStages]), static_cast<uint32_t>(kb / kStages) & 1u)) ok = false;
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {
      for (int32_t kb = 0; kb < ro.kblocks; ++kb) {
        const int s = kb % kStages;
        const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
        if (!mbar_wait(smem_u32(&bars[kStages + s]), ph)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = smem_u32(base + s * L::kBytes);
        const uint32_t a_hi = st + L::kAhi, a_lo = st + L::kAlo, b_hi = st + L::kBhi, b_lo = st + L::kBlo;
        if constexpr (BF16) {
#pragma unroll
          for (int kk = 0; kk < kBK / 16; ++kk) {
            const uint32_t off = kk * 32;  // 16 bfloat16 of K inside the 64-byte swizzled row
            mma_bf16(tmem, sw64_desc(a_hi + off), sw64_desc(b_hi + off), (kb | kk) != 0);
            mma_bf16(tmem, sw64_desc(a_hi + off), sw64_desc(b_lo + off), 1u);
            mma_bf16(tmem, sw64_desc(a_lo + off), sw64_desc(b_hi + off), 1u);
          }
        } else {
#pragma unroll
          for (int kk = 0; kk < kBK / 8; ++kk) {
            const uint32_t off = kk * 32;  // 8 tf32 of K inside the 128-byte swizzled row
            mma_tf32(tmem, sw128_desc(a_hi + off), sw128_desc(b_hi + off), (kb | kk) != 0);
            mma_tf32(tmem, sw128_desc(a_hi + off), sw128_desc(b_lo + off), 1u);
            mma_tf32(tmem, sw128_desc(a_lo + off), sw128_desc(b_hi + off), 1u);
          }
        }
        mma_commit(smem_u32(&bars[2 * kStages + s]));
      }
      mma_commit(smem_u32(&bars[3 * kStages]));
    }
  } else {
    // warps 0-3: split the A tile of every stage, then the epilogue
    const int t = threadIdx.x;  // 0..127
    for (int32_t kb = 0; kb < ro.kblocks; ++kb) {
      const int s = kb % kStages;
      const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
      if (!mbar_wait(smem_u32(&bars[s]), ph)) {
        ok = false;
        break;
      }
      unsigned char* st = base + s * L::kBytes;
      float4* a = reinterpret_cast<float4*>(st);
      if constexpr (BF16) {
        // the float32 tile (128-byte rows, 16-byte unit u of row r at unit u ^ (r & 7)) into the hi
        // and lo bfloat16 tiles (64-byte rows, 16-byte unit u of row r at unit u ^ ((r >> 1) & 3))
#pragma unroll
        for (int i = 0; i < L::kTileF32 / 16 / 128; ++i) {
          const int idx = t + 128 * i;  // the physical float4 of the float32 tile
          const int r = idx >> 3;
          const int k0 = ((idx & 7) ^ (r & 7)) * 4;  // its first K column
          const float4 v = a[idx];
          const float f[4] = {v.x, v.y, v.z, v.w};
          uint32_t hb[4], lb[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            hb[q] = bf16_bits(f[q]);
            lb[q] = bf16_bits(__fsub_rn(f[q], bf16_value(hb[q])));
          }
          const int at = r * 64 + ((((k0 >> 3) ^ ((r >> 1) & 3))) << 4) + ((k0 & 7) << 1);
          *reinterpret_cast<uint2*>(st + L::kAhi + at) = make_uint2(hb[0] | (hb[1] << 16), hb[2] | (hb[3] << 16));
          *reinterpret_cast<uint2*>(st + L::kAlo + at) = make_uint2(lb[0] | (lb[1] << 16), lb[2] | (lb[3] << 16));
        }
      } else {
        float4* alo = reinterpret_cast<float4*>(st + L::kAlo);
#pragma unroll
        for (int i = 0; i < L::kTileF32 / 16 / 128; ++i) {
          const int idx = t + 128 * i;
          const float4 v = a[idx];
          float4 h, l;
          h.x = to_tf32(v.x);
          h.y = to_tf32(v.y);
          h.z = to_tf32(v.z);
          h.w = to_tf32(v.w);
          l.x = to_tf32(__fsub_rn(v.x, h.x));
          l.y = to_tf32(__fsub_rn(v.y, h.y));
          l.z = to_tf32(__fsub_rn(v.z, h.z));
          l.w = to_tf32(__fsub_rn(v.w, h.w));
          a[idx] = h;
          alo[idx] = l;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(smem_u32(&bars[kStages + s]));
    }
    // the tcgen05.ld below is warp-collective: the warp decides together
    const bool acc_ready = __all_sync(0xffffffffu, ok && mbar_wait(smem_u32(&bars[3 * kStages]), 0));
    if (acc_ready) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int64_t m = m0 + warp * 32 + lane;
      bool valid = m < ro.M;
      int64_t obase = 0;
      if (valid) {
        const int64_t b = m / ro.rows, r = m - b * ro.rows;
        const int64_t hi = r / ro.n_lo, lo = r - hi * ro.n_lo;
        valid = run[b] != 0;
        obase = b * ro.f_out + hi * ro.pitch_out + lo;
      }
#pragma unroll 1
      for (int c = 0; c < kBN / 32; ++c) {
        float v[32];
        tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c * 32), v);
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < 32; ++jj) {
            const int32_t j = n0 + c * 32 + jj;
            if (j < ro.N) out[obase + static_cast<int64_t>(j) * ro.s_j] = v[jj];
          }
        }
      }
    } else {
      ok = false;
    }
  }
  if (!ok) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 5) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN) : "memory");
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess) {
      fn = reinterpret_cast<EncodeTiled>(p);
    }
    (void)cudaGetLastError();
  });
  if (!fn) throw CudaError("eda: cuTensorMapEncodeTiled is unavailable", static_cast<int>(cudaErrorNotSupported));
  return fn;
}

// A 2-D tensor map of float32 (128-byte swizzle) or bfloat16 (64-byte swizzle) elements: inner
// extent `inner` (contiguous), `outer` rows `stride` elements apart, boxes of 32 x box_rows
// elements (one swizzled row each); reads past the extents return zeros.
CUtensorMap make_map(const void* base, bool bf16, uint64_t inner, uint64_t outer, uint64_t stride, uint32_t box_rows) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof m);
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {stride * (bf16 ? 2 : 4)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                                 const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 bf16 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    throw CudaError("eda: cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")",
                    static_cast<int>(cudaErrorInvalidValue));
  }
  return m;
}

template <bool BF16>
void set_smem_once() {
  once_on_device(reinterpret_cast<const void*>(gemm_tc<BF16>), [] {
    EDAB_CUDA(cudaFuncSetAttribute(gemm_tc<BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, Stage<BF16>::kSmem));
  });
}

}  // namespace tc

// One rotated axis pass on the tensor cores (orient.cuh): see RotPass.
void rot_pass_tc(cudaStream_t s, const RotPass& p, const void* basis, bool bf16, int32_t kpad, int32_t npad,
                 const float* in, float* out, const int32_t* run, int32_t* err) {
  if (p.M < 1) return;
  const CUtensorMap ta = tc::make_map(in, false, static_cast<uint64_t>(p.K), static_cast<uint64_t>(p.M),
                                      static_cast<uint64_t>(p.pitch_in), tc::kBM);
  const CUtensorMap tb = tc::make_map(basis, bf16, static_cast<uint64_t>(kpad), static_cast<uint64_t>(2 * npad),
                                      static_cast<uint64_t>(kpad), tc::kBN);
  tc::RotOut ro{};
  ro.M = p.M;
  ro.N = p.K;
  ro.kblocks = (p.K + tc::kBK - 1) / tc::kBK;
  ro.npad = npad;
  ro.rows = p.rows;
  ro.n_lo = p.n_lo;
  ro.pitch_out = p.pitch_out;
  ro.s_j = p.s_j;
  ro.f_out = p.f_out;
  const int64_t mt = (p.M + tc::kBM - 1) / tc::kBM;
  if (mt > 0x7fffffffLL) throw std::invalid_argument("eda: orientation pass too large");
  const dim3 grid(static_cast<unsigned>((p.K + tc::kBN - 1) / tc::kBN), static_cast<unsigned>(mt));
  if (bf16) {
    tc::set_smem_once<true>();
    tc::gemm_tc<true><<<grid, tc::kThreadsTc, tc::Stage<true>::kSmem, s>>>(ta, tb, ro, out, run, err);
  } else {
    tc::set_smem_once<false>();
    tc::gemm_tc<false><<<grid, tc::kThreadsTc, tc::Stage<false>::kSmem, s>>>(ta, tb, ro, out, run, err);
  }
  EDAB_LAUNCH("gemm_tc");
}

}  // namespace edab
