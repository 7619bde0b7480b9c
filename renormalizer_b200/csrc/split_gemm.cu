// Split-precision complex GEMM on the 5th-generation tensor cores (sm_100a).
//
// C (real or complex) = opA(A) opB(B) with A, B real or complex with any
// strides, computed as
//     A ~ A_hi + A_lo,  B ~ B_hi + B_lo    (BF16 or TF32 pairs)
//     C ~ A_hi B_hi + A_hi B_lo + A_lo B_hi   (FP32 accumulation in TMEM)
// Complex operands use the real embedding: the smaller operand is "doubled"
// into [[Re, -Im], [Im, Re]] rows, the other is K-concatenated as [Re | Im],
// so each complex GEMM is ONE real GEMM whose rows (or columns) interleave the
// real and imaginary parts of the result.
//
// Pipeline (persistent: one CTA per SM walks 128 x 256 output tiles; 10 warps):
//   warp 0     TMA producer: 4 tiles per stage (A_hi, A_lo, B_hi, B_lo),
//              128-byte swizzled K-major boxes, mbarrier complete_tx
//   warp 1     TMEM allocator + single-thread tcgen05.mma issuer: 3 products
//              per stage, tcgen05.commit frees the stage
//   warps 2-9  epilogue (two warps per TMEM lane quarter, half the columns
//              each): tcgen05.ld 32x32b from TMEM, strided writes of the
//              (interleaved complex) output as FP64, or as FP32 when the
//              output only feeds the next split stage (the accumulator is
//              FP32, so nothing is lost) -- the operands A, B are FP64 or
//              such FP32 intermediates
// Every mbarrier wait is bounded; on timeout the kernel records the site in
// a device error word, skips the remaining work and still frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstring>
#include "split_gemm.cuh"

namespace reno {
namespace split {

constexpr int BM = 128, BN = 256, STAGES = 2, THREADS = 320;  // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int EPI_WARPS = 8;
constexpr int KROW_BYTES = 128;  // one SW128 row of K per stage
constexpr int A_TILE = BM * KROW_BYTES;   // 16 KB
constexpr int B_TILE = BN * KROW_BYTES;   // 32 KB
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr uint32_t TMEM_COLS = 256;  // one accumulator buffer (two are allocated)

// device error word: 0 = ok; otherwise 1000 + site of the first timed-out wait
__device__ int g_split_error = 0;

enum OutMode { OUT_REAL = 0, OUT_COLS_CPLX = 1, OUT_ROWS_CPLX = 2, OUT_PACK = 3 };

struct Epi {
  void* C;
  int64_t sCm, sCn, sCb;  // output strides in output elements
  int M, N;               // logical output dims
  int mode;
  int accumulate;
  int rows_p, cols_p;     // rows / cols of the real product C' actually present
  int c_f32;              // C holds float (complex: float2) instead of double
  // OUT_PACK: the tile is written as the next split stage's packed operand.
  // Output element (m, n, ri) of the real product (ri: re/im component, from
  // the row interleave when A was doubled, inter = 1, or the column interleave
  // when B was doubled, inter = 2) goes to hi/lo element
  //   bz*s_b + (m / Dm)*s_m1 + (m % Dm)*s_m0 + (n / Dn)*s_n1 + (n % Dn)*s_n0 + ri*s_ri
  void* phi;
  void* plo;
  int64_t s_b, s_m1, s_m0, s_n1, s_n0, s_ri;
  int Dm, Dn, inter;
};

template <typename T>
__device__ __forceinline__ void st_real(void* C, int64_t i, float v, int acc) {
  T* p = reinterpret_cast<T*>(C) + i;
  *p = (acc ? *p : T(0)) + (T)v;
}

template <typename T2>
__device__ __forceinline__ void st_cplx(void* C, int64_t i, float re, float im, int acc) {
  T2* p = reinterpret_cast<T2*>(C) + i;
  T2 o = acc ? *p : T2{0, 0};
  o.x += re;
  o.y += im;
  *p = o;
}

// x = hi + lo in the split format: bits of hi and lo (BF16 in the low 16 bits, or TF32)
template <int ESZ>
__device__ __forceinline__ void split_bits(float x, uint32_t& hb, uint32_t& lb) {
  if constexpr (ESZ == 2) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hb = __bfloat16_as_ushort(h);
    lb = __bfloat16_as_ushort(l);
  } else {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(x));
    const float rem = x - __uint_as_float(hb);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lb) : "f"(rem));
  }
}

template <int ESZ>
__device__ __forceinline__ void split_store_bits(void* hi, void* lo, int64_t idx, uint32_t hb, uint32_t lb) {
  if constexpr (ESZ == 2) {
    reinterpret_cast<unsigned short*>(hi)[idx] = (unsigned short)hb;
    reinterpret_cast<unsigned short*>(lo)[idx] = (unsigned short)lb;
  } else {
    reinterpret_cast<uint32_t*>(hi)[idx] = hb;
    reinterpret_cast<uint32_t*>(lo)[idx] = lb;
  }
}

// 16 output values v[t*STRIDE + OFF] (t = 0..15) of one (m, ri) for columns
// n0 .. n0+15 into the packed planes: one 32-byte (BF16) or 64-byte (TF32)
// vector store per plane when the run is contiguous and aligned, scalar
// stores otherwise
template <int ESZ, int STRIDE, int OFF>
__device__ __forceinline__ void pack_run(const float* v, const Epi& e, int64_t mbase, int n0, int ri) {
  const int64_t rbase = mbase + (int64_t)ri * e.s_ri;
  const int64_t idx0 = rbase + (int64_t)(n0 / e.Dn) * e.s_n1 + (int64_t)(n0 % e.Dn) * e.s_n0;
  const bool vec = e.s_n0 == 1 && n0 + 16 <= e.N && (n0 % e.Dn) + 16 <= e.Dn && (idx0 % (16 / ESZ)) == 0;
  if (vec) {
    uint32_t hb[16], lb[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) split_bits<ESZ>(v[t * STRIDE + OFF], hb[t], lb[t]);
    if constexpr (ESZ == 2) {
      uint4* ph = reinterpret_cast<uint4*>(reinterpret_cast<unsigned short*>(e.phi) + idx0);
      uint4* pl = reinterpret_cast<uint4*>(reinterpret_cast<unsigned short*>(e.plo) + idx0);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        ph[q] = make_uint4(hb[8 * q] | (hb[8 * q + 1] << 16), hb[8 * q + 2] | (hb[8 * q + 3] << 16),
                           hb[8 * q + 4] | (hb[8 * q + 5] << 16), hb[8 * q + 6] | (hb[8 * q + 7] << 16));
        pl[q] = make_uint4(lb[8 * q] | (lb[8 * q + 1] << 16), lb[8 * q + 2] | (lb[8 * q + 3] << 16),
                           lb[8 * q + 4] | (lb[8 * q + 5] << 16), lb[8 * q + 6] | (lb[8 * q + 7] << 16));
      }
    } else {
      uint4* ph = reinterpret_cast<uint4*>(reinterpret_cast<uint32_t*>(e.phi) + idx0);
      uint4* pl = reinterpret_cast<uint4*>(reinterpret_cast<uint32_t*>(e.plo) + idx0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        ph[q] = make_uint4(hb[4 * q], hb[4 * q + 1], hb[4 * q + 2], hb[4 * q + 3]);
        pl[q] = make_uint4(lb[4 * q], lb[4 * q + 1], lb[4 * q + 2], lb[4 * q + 3]);
      }
    }
  } else {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int n = n0 + t;
      if (n < e.N) {
        uint32_t hb, lb;
        split_bits<ESZ>(v[t * STRIDE + OFF], hb, lb);
        split_store_bits<ESZ>(e.phi, e.plo, rbase + (int64_t)(n / e.Dn) * e.s_n1 + (int64_t)(n % e.Dn) * e.s_n0,
                              hb, lb);
      }
    }
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait (wait_ns of wall clock): returns false and raises the abort flag on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int site,
                                          uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255u) == 255u) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > wait_ns) break;
    }
  }
  *abort_flag = 1;
  atomicCAS(&g_split_error, 0, 1000 + site);
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (SBO = 8 rows x 128 B)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1u << 46;            // descriptor version for sm_100
  d |= (uint64_t)2u << 61;            // SWIZZLE_128B
  return d;
}

template <int ESZ>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  if constexpr (ESZ == 2) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
  }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

#define TMEM_LD32(taddr, r)                                                                                         \
  asm volatile(                                                                                                     \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18," \
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                                                \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),            \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),      \
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),    \
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])     \
      : "r"(taddr))

// Epilogue of columns [c_begin, c_end) of one output tile: TMEM -> registers
// (32 columns at a time) -> the output in the Epi mode.  Warp w reads TMEM
// lane quarter q = w % 4, i.e. tile rows q*32 .. q*32+31; two warps share a
// quarter, each taking half of the BN columns.
// Output of 32 accumulated columns c0 .. c0+31 of tile row q*32 + lane in the
// Epi mode.
template <int ESZ>
__device__ __forceinline__ void epilogue_store(const Epi& epi, const float* v, int q, int lane, int m_tile, int n_tile,
                                               int bz, int c0) {
  const int row = q * 32 + lane;  // tile row of this thread
  const int rp = m_tile * BM + row;
  {
    const int cp = n_tile * BN + c0;  // product column of v[0]
    if (epi.mode == OUT_PACK) {
      const int m = epi.inter == 1 ? (rp >> 1) : rp;
      if (m < epi.M) {
        const int64_t mbase =
            (int64_t)bz * epi.s_b + (int64_t)(m / epi.Dm) * epi.s_m1 + (int64_t)(m % epi.Dm) * epi.s_m0;
        if (epi.inter == 2) {
          pack_run<ESZ, 2, 0>(v, epi, mbase, cp / 2, 0);
          pack_run<ESZ, 2, 1>(v, epi, mbase, cp / 2, 1);
        } else {
          const int ri = epi.inter == 1 ? (rp & 1) : 0;
          pack_run<ESZ, 1, 0>(v, epi, mbase, cp, ri);
          pack_run<ESZ, 1, 16>(v, epi, mbase, cp + 16, ri);
        }
      }
    } else if (epi.mode == OUT_REAL) {
      if (rp < epi.M) {
        const int64_t base = (int64_t)bz * epi.sCb + (int64_t)rp * epi.sCm;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = cp + j;
          if (n < epi.N) {
            if (epi.c_f32)
              st_real<float>(epi.C, base + (int64_t)n * epi.sCn, v[j], epi.accumulate);
            else
              st_real<double>(epi.C, base + (int64_t)n * epi.sCn, v[j], epi.accumulate);
          }
        }
      }
    } else if (epi.mode == OUT_COLS_CPLX) {
      if (rp < epi.M) {
        const int64_t base = (int64_t)bz * epi.sCb + (int64_t)rp * epi.sCm;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = cp / 2 + j;
          if (n < epi.N) {
            if (epi.c_f32)
              st_cplx<float2>(epi.C, base + (int64_t)n * epi.sCn, v[2 * j], v[2 * j + 1], epi.accumulate);
            else
              st_cplx<double2>(epi.C, base + (int64_t)n * epi.sCn, v[2 * j], v[2 * j + 1], epi.accumulate);
          }
        }
      }
    } else {
      // rows interleave re/im: lanes (2i, 2i+1) hold (re, im) of complex row rp/2
      const bool even = (lane & 1) == 0;
      float mine[16], got[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float send = even ? v[16 + j] : v[j];
        got[j] = __shfl_xor_sync(0xffffffffu, send, 1);
        mine[j] = even ? v[j] : v[16 + j];
      }
      const int m = rp >> 1;
      if (m < epi.M) {
        const int64_t base = (int64_t)bz * epi.sCb + (int64_t)m * epi.sCm;
        const int nb = cp + (even ? 0 : 16);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = nb + j;
          if (n < epi.N) {
            const float re = even ? mine[j] : got[j], im = even ? got[j] : mine[j];
            if (epi.c_f32)
              st_cplx<float2>(epi.C, base + (int64_t)n * epi.sCn, re, im, epi.accumulate);
            else
              st_cplx<double2>(epi.C, base + (int64_t)n * epi.sCn, re, im, epi.accumulate);
          }
        }
      }
    }
  }
}

template <int ESZ>
__device__ __forceinline__ void epilogue_tile(const Epi& epi, uint32_t tacc, int q, int lane, int m_tile, int n_tile,
                                              int bz, int c_begin, int c_end) {
  for (int c0 = c_begin; c0 < c_end; c0 += 32) {
    uint32_t r[32];
    const uint32_t taddr = tacc + ((uint32_t)(q * 32) << 16) + (uint32_t)c0;
    TMEM_LD32(taddr, r);
    asm volatile("tcgen05.wait::ld.sync.aligned;");
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
    epilogue_store<ESZ>(epi, v, q, lane, m_tile, n_tile, bz, c0);
  }
}

// tile t of the (bz, slow, fast) raster: M tiles fastest when m_fast
__device__ __forceinline__ void tile_coords(int t, int mt, int nt, int m_fast, int& m_tile, int& n_tile, int& bz) {
  const int per = mt * nt;
  bz = t / per;
  const int r = t - bz * per;
  if (m_fast) {
    m_tile = r % mt;
    n_tile = r / mt;
  } else {
    n_tile = r % nt;
    m_tile = r / nt;
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait that ignores the abort flag: used only to drain the CTA's own
// copies and MMAs in flight before it frees TMEM and exits
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity, uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(bar, parity)) return;
    if ((it & 255u) == 255u && global_ns() - t0 > wait_ns) {
      atomicCAS(&g_split_error, 0, 1009);
      return;
    }
  }
}

// Persistent kernel: one CTA per SM walks output tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... in the raster above.  TMEM holds two BN-column
// FP32 accumulators; the MMA thread fills buffer (i & 1) for the CTA's i-th
// tile while the epilogue warps drain the other, so each tile's epilogue
// overlaps the next tile's TMA + MMA mainloop.  The smem stage ring runs on
// across tiles.  Barriers: full / empty (TMA <-> MMA, per stage), tmem_full
// (MMA -> epilogue, per buffer, tcgen05.commit), tmem_empty (epilogue -> MMA,
// per buffer, one arrive per epilogue warp, 8 warps), drain (the MMA thread's last
// commit, waited for before TMEM is freed).
//
// PROMOTE (opt-in, reno_set_split_accumulation_chunk): the tensor cores'
// FP32 accumulation truncates, so its error is a bias that grows with the
// number of terms.  In this form a tile's K range is cut into chunks of kc K
// tiles; each chunk accumulates in one TMEM buffer (the two buffers
// alternate chunk by chunk, so the MMA fills one while the epilogue reads the
// other), and the epilogue warps add every chunk's partial sums into FP32
// registers with round-to-nearest additions before the tile's output.
template <int ESZ, bool PROMOTE>
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                      const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl, Epi epi,
                      int num_k_tiles, int k_elems, int a_batched, int b_batched, int m_fast, int mt, int nt,
                      int ntiles, uint64_t wait_ns, int skip_stage, int kc) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tmem_full = empty + STAGES;  // [2]
  uint64_t* tmem_empty = tmem_full + 2;  // [2]
  uint64_t* drain = tmem_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tmem_full[b], 1);
      mbar_init(&tmem_empty[b], EPI_WARPS);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    uint32_t g = 0;  // k tiles issued by this CTA
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      int m_tile, n_tile, bz;
      tile_coords(t, mt, nt, m_fast, m_tile, n_tile, bz);
      const int za = a_batched ? bz : 0, zb = b_batched ? bz : 0;
      for (int kt = 0; kt < num_k_tiles; ++kt) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1;
        if (!mbar_wait(&empty[s], ph ^ 1, abort_flag, 1, wait_ns)) {
          ok = false;
          break;
        }
        if (blockIdx.x == 0 && (int)g == skip_stage) {  // test hook: stage g of CTA 0 stays unloaded
          ++g;
          continue;
        }
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        const int kx = kt * (KROW_BYTES / ESZ);
        tma_load_3d(st, &tmAh, &full[s], kx, m_tile * BM, za);
        tma_load_3d(st + A_TILE, &tmAl, &full[s], kx, m_tile * BM, za);
        tma_load_3d(st + 2 * A_TILE, &tmBh, &full[s], kx, n_tile * BN, zb);
        tma_load_3d(st + 2 * A_TILE + B_TILE, &tmBl, &full[s], kx, n_tile * BN, zb);
        ++g;
      }
    }
    // land every copy this CTA issued before it can exit (immediate for the
    // ones the MMA thread already consumed)
    for (uint32_t j = (g > (uint32_t)STAGES ? g - STAGES : 0u); j < g; ++j)
      mbar_drain(&full[j % STAGES], (j / STAGES) & 1, wait_ns);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    constexpr uint32_t fmt = ESZ == 2 ? 1u : 2u;  // BF16 : TF32
    const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    uint32_t g = 0;
    bool ok = true;
    int i = 0;  // accumulation units: tiles, or (tile, chunk) pairs under PROMOTE
    const int chunk = PROMOTE ? kc : num_k_tiles;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x)
     for (int k0 = 0; k0 < num_k_tiles && ok; k0 += chunk, ++i) {
      const int b = i & 1;
      const uint32_t use = (uint32_t)(i >> 1);
      if (!mbar_wait(&tmem_empty[b], (use & 1) ^ 1, abort_flag, 4, wait_ns)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t tacc = tmem + (uint32_t)(b * TMEM_COLS);
      const int k1 = min(num_k_tiles, k0 + chunk);
      for (int kt = k0; kt < k1; ++kt) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1;
        if (!mbar_wait(&full[s], ph, abort_flag, 2, wait_ns)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
        const uint64_t dah = sdesc(base), dal = sdesc(base + A_TILE);
        const uint64_t dbh = sdesc(base + 2 * A_TILE), dbl = sdesc(base + 2 * A_TILE + B_TILE);
        // K beyond k_elems is TMA zero fill: skip the sub-steps that only see it
        constexpr int SUB = (KROW_BYTES / ESZ) / 4;  // elements per 32-byte instruction step
        const int rem = k_elems - kt * (KROW_BYTES / ESZ);
        const int nsub = rem >= 4 * SUB ? 4 : (rem + SUB - 1) / SUB;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          if (kk < nsub) {
            const uint64_t adv = (uint64_t)((kk * 32) >> 4);  // 32 bytes of K per instruction
            const uint32_t first = (kt == k0 && kk == 0) ? 0u : 1u;
            umma<ESZ>(tacc, dah + adv, dbh + adv, idesc, first);
            umma<ESZ>(tacc, dah + adv, dbl + adv, idesc, 1u);
            umma<ESZ>(tacc, dal + adv, dbh + adv, idesc, 1u);
          }
        }
        umma_commit(&empty[s]);
        ++g;
      }
      if (ok) umma_commit(&tmem_full[b]);
    }
    // every MMA this thread issued completes before TMEM is freed
    umma_commit(drain);
    mbar_drain(drain, 0, wait_ns);
  } else if (warp >= 2) {
    // ---------------- epilogue
    const int q = warp % 4;                      // TMEM lane quarter this warp may access
    const int c_begin = ((warp - 2) / 4) * (BN / 2);  // warps 2-5: columns [0, BN/2), warps 6-9: the rest
    int i = 0;
    if constexpr (PROMOTE) {
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        float acc[BN / 2];  // this thread's row, columns c_begin .. c_begin + BN/2 - 1
        for (int k0 = 0; k0 < num_k_tiles; k0 += kc, ++i) {
          const int b = i & 1;
          const uint32_t use = (uint32_t)(i >> 1);
          if (!mbar_wait(&tmem_full[b], use & 1, abort_flag, 3, wait_ns) || *abort_flag) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t tacc = tmem + (uint32_t)(b * TMEM_COLS) + ((uint32_t)(q * 32) << 16) + (uint32_t)c_begin;
#pragma unroll
          for (int p = 0; p < BN / 64; ++p) {
            uint32_t r[32];
            TMEM_LD32(tacc + (uint32_t)(32 * p), r);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int j = 0; j < 32; ++j)
              acc[32 * p + j] = k0 == 0 ? __uint_as_float(r[j]) : __fadd_rn(acc[32 * p + j], __uint_as_float(r[j]));
          }
          asm volatile("tcgen05.fence::before_thread_sync;");
          __syncwarp();
          if (lane == 0) mbar_arrive(&tmem_empty[b]);
        }
        if (!ok) break;
        int m_tile, n_tile, bz;
        tile_coords(t, mt, nt, m_fast, m_tile, n_tile, bz);
#pragma unroll
        for (int p = 0; p < BN / 64; ++p) epilogue_store<ESZ>(epi, acc + 32 * p, q, lane, m_tile, n_tile, bz, c_begin + 32 * p);
      }
    } else {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
      const int b = i & 1;
      const uint32_t use = (uint32_t)(i >> 1);
      if (!mbar_wait(&tmem_full[b], use & 1, abort_flag, 3, wait_ns)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (*abort_flag) break;
      int m_tile, n_tile, bz;
      tile_coords(t, mt, nt, m_fast, m_tile, n_tile, bz);
      epilogue_tile<ESZ>(epi, tmem + (uint32_t)(b * TMEM_COLS), q, lane, m_tile, n_tile, bz, c_begin,
                         c_begin + BN / 2);
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tmem_empty[b]);
    }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TMEM_COLS));
  }
}

// ------------------------------------------------------------------ packing
// Operand packing modes (rows R, reduction length K of the logical operand):
enum PackMode {
  P_REAL = 0,       // out[r][k]       = x[r,k]                       K' = K
  P_CAT = 1,        // out[r][k | K+k] = (re, im) of x[r,k]           K' = 2K
  P_DBL_CPLX = 2,   // out[2r] = [re, -im], out[2r+1] = [im, re]      K' = 2K, 2R rows
  P_DBL_SPLIT = 3   // out[2r][k] = re, out[2r+1][k] = im             K' = K,  2R rows
};

struct PackArgs {
  const void* src;
  int src_complex, conj, src_f32;
  int64_t s_r, s_k, s_b;  // element strides of rows, K and batch
  // row r = (r2 * D1 + r1) * D0 + r0 sits at r0*s_r + r1*s_r1 + r2*s_r2
  // (a single-strided row index has D0 >= R)
  int D0, D1;
  int64_t s_r1, s_r2;
  int R, K, nbatch, mode;
  void* hi;
  void* lo;
  int64_t pitch;        // row pitch of the packed buffer (elements, 16-byte multiple)
  int64_t rows_out;     // rows per batch in the packed buffer
};

template <int ESZ>
__device__ __forceinline__ void split_store(void* hi, void* lo, int64_t idx, double x) {
  if constexpr (ESZ == 2) {
    const __nv_bfloat16 h = __double2bfloat16(x);
    const __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
    reinterpret_cast<__nv_bfloat16*>(hi)[idx] = h;
    reinterpret_cast<__nv_bfloat16*>(lo)[idx] = l;
  } else {
    const float f = (float)x;
    uint32_t hb, lb;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(f));
    const float h = __uint_as_float(hb);
    const float rem = (float)(x - (double)h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lb) : "f"(rem));
    reinterpret_cast<float*>(hi)[idx] = h;
    reinterpret_cast<float*>(lo)[idx] = __uint_as_float(lb);
  }
}

// one 32 x 32 (rows x K) source tile per block, staged through shared memory so
// that both the strided reads (FP64, or FP32 intermediates) and the
// K-contiguous packed writes coalesce.  Packed rows hold K' elements at a
// 16-byte pitch; the tensor maps end at K', so the TMA loads zero-fill the
// rest of the last 128-byte K tile and no padding is ever written.
template <int ESZ>
__global__ void pack_kernel(PackArgs a) {
  __shared__ double2 tile[32][33];
  const int b = blockIdx.z;
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const bool k_fast = (a.s_k == 1) || (a.s_r != 1);
  for (int i = ty; i < 32; i += 8) {
    const int r = k_fast ? r0 + i : r0 + tx;
    const int k = k_fast ? k0 + tx : k0 + i;
    double2 v = make_double2(0.0, 0.0);
    if (r < a.R && k < a.K) {
      const int r0 = r % a.D0, rq = r / a.D0;
      const int64_t roff = (int64_t)r0 * a.s_r + (int64_t)(rq % a.D1) * a.s_r1 + (int64_t)(rq / a.D1) * a.s_r2;
      const int64_t off = (int64_t)b * a.s_b + roff + (int64_t)k * a.s_k;
      if (a.src_complex) {
        if (a.src_f32) {
          const float2 f = reinterpret_cast<const float2*>(a.src)[off];
          v = make_double2(f.x, f.y);
        } else {
          v = reinterpret_cast<const double2*>(a.src)[off];
        }
        if (a.conj) v.y = -v.y;
      } else {
        v.x = a.src_f32 ? (double)reinterpret_cast<const float*>(a.src)[off] : reinterpret_cast<const double*>(a.src)[off];
      }
    }
    if (k_fast)
      tile[i][tx] = v;
    else
      tile[tx][i] = v;
  }
  __syncthreads();
  const int64_t base = (int64_t)b * a.rows_out * a.pitch;
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i, k = k0 + tx;
    if (r >= a.R) continue;
    const double2 v = tile[i][tx];
    const bool kin = k < a.K;
    switch (a.mode) {
      case P_REAL:
        if (kin) split_store<ESZ>(a.hi, a.lo, base + (int64_t)r * a.pitch + k, v.x);
        break;
      case P_CAT:
        if (kin) {
          split_store<ESZ>(a.hi, a.lo, base + (int64_t)r * a.pitch + k, v.x);
          split_store<ESZ>(a.hi, a.lo, base + (int64_t)r * a.pitch + a.K + k, v.y);
        }
        break;
      case P_DBL_CPLX:
        if (kin) {
          const int64_t r2 = base + (int64_t)(2 * r) * a.pitch;
          split_store<ESZ>(a.hi, a.lo, r2 + k, v.x);
          split_store<ESZ>(a.hi, a.lo, r2 + a.K + k, -v.y);
          split_store<ESZ>(a.hi, a.lo, r2 + a.pitch + k, v.y);
          split_store<ESZ>(a.hi, a.lo, r2 + a.pitch + a.K + k, v.x);
        }
        break;
      default:  // P_DBL_SPLIT
        if (kin) {
          const int64_t r2 = base + (int64_t)(2 * r) * a.pitch;
          split_store<ESZ>(a.hi, a.lo, r2 + k, v.x);
          split_store<ESZ>(a.hi, a.lo, r2 + a.pitch + k, v.y);
        }
        break;
    }
  }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the driver's tensor-map encoder, fetched through the runtime so that the
// library does not link libcuda (it loads on machines without a driver)
static EncodeTiledFn encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 3-D map (K', rows, batch) over a packed buffer of row pitch `pitch`; loads
// past K' read zeros
static bool make_map(CUtensorMap* tm, void* base, int esz, int64_t kext, int64_t pitch, int64_t rows, int64_t nb,
                     int box_rows) {
  EncodeTiledFn enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {(cuuint64_t)kext, (cuuint64_t)rows, (cuuint64_t)nb};
  cuuint64_t strides[2] = {(cuuint64_t)(pitch * esz), (cuuint64_t)(pitch * esz * rows)};
  cuuint32_t box[3] = {(cuuint32_t)(KROW_BYTES / esz), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(tm, esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims,
                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

struct Plan {
  int esz, kstep;        // element size, elements per 128-byte K row
  int modeA, modeB, out;
  int64_t KA;            // logical K' (after re/im concatenation)
  int64_t pitch;         // packed row pitch: K' rounded up to 16 bytes
  int64_t rowsA, rowsB;  // packed rows per batch
  int64_t nbA, nbB;      // packed batches
  size_t offAh, offAl, offBh, offBl, total;
};

static size_t al(size_t x) { return (x + 1023) & ~size_t(1023); }

static Plan make_plan(const GemmParams& p, int prec) {
  Plan q{};
  q.esz = prec == RENO_PREC_BF16X3 ? 2 : 4;
  q.kstep = KROW_BYTES / q.esz;
  const bool ac = p.A.is_complex, bc = p.B.is_complex;
  int64_t kf = 1;
  if (ac && bc) {
    // double the operand with fewer rows: its rows are re-used across the whole other side
    const bool dblA = (int64_t)p.M * (p.A.s_batch ? p.batch : 1) <= (int64_t)p.N * (p.B.s_batch ? p.batch : 1);
    if (dblA) {
      q.modeA = P_DBL_CPLX;
      q.modeB = P_CAT;
      q.out = OUT_ROWS_CPLX;
    } else {
      q.modeA = P_CAT;
      q.modeB = P_DBL_CPLX;
      q.out = OUT_COLS_CPLX;
    }
    kf = 2;
  } else if (bc) {
    q.modeA = P_REAL;
    q.modeB = P_DBL_SPLIT;
    q.out = OUT_COLS_CPLX;
  } else if (ac) {
    q.modeA = P_DBL_SPLIT;
    q.modeB = P_REAL;
    q.out = OUT_ROWS_CPLX;
  } else {
    q.modeA = P_REAL;
    q.modeB = P_REAL;
    q.out = OUT_REAL;
  }
  q.KA = kf * p.K;
  const int64_t align = 16 / q.esz;  // TMA row strides are 16-byte multiples
  q.pitch = ((q.KA + align - 1) / align) * align;
  q.rowsA = (q.modeA == P_DBL_CPLX || q.modeA == P_DBL_SPLIT) ? 2 * (int64_t)p.M : p.M;
  q.rowsB = (q.modeB == P_DBL_CPLX || q.modeB == P_DBL_SPLIT) ? 2 * (int64_t)p.N : p.N;
  q.nbA = p.A.s_batch ? p.batch : 1;
  q.nbB = p.B.s_batch ? p.batch : 1;
  const size_t sa = (size_t)q.rowsA * q.pitch * q.nbA * q.esz;
  const size_t sb = (size_t)q.rowsB * q.pitch * q.nbB * q.esz;
  q.offAh = 0;
  q.offAl = al(sa);
  q.offBh = q.offAl + al(sa);
  q.offBl = q.offBh + al(sb);
  q.total = q.offBl + al(sb);
  return q;
}

template <int ESZ>
static cudaError_t run_pack(const GemmOperand& op, int R, int K, int nb, int mode, const SplitRows& rs, void* hi,
                            void* lo, int64_t pitch, int64_t rows_out, cudaStream_t st) {
  PackArgs a;
  a.src = op.ptr;
  a.src_complex = op.is_complex;
  a.conj = op.conj;
  a.src_f32 = op.is_f32;
  a.s_r = op.s_outer;
  a.s_k = op.s_k;
  a.s_b = op.s_batch;
  a.D0 = rs.D0 > 0 ? rs.D0 : std::max(R, 1);
  a.D1 = rs.D0 > 0 ? std::max(rs.D1, 1) : 1;
  a.s_r1 = rs.D0 > 0 ? rs.s_r1 : 0;
  a.s_r2 = rs.D0 > 0 ? rs.s_r2 : 0;
  a.R = R;
  a.K = K;
  a.nbatch = nb;
  a.mode = mode;
  a.hi = hi;
  a.lo = lo;
  a.pitch = pitch;
  a.rows_out = rows_out;
  dim3 grid((unsigned)ceil_div(K, 32), (unsigned)ceil_div(R, 32), (unsigned)nb);
  count_launch();
  pack_kernel<ESZ><<<grid, dim3(32, 8), 0, st>>>(a);
  return cudaGetLastError();
}

static int inter_of(int modeA, int modeB) {
  if (modeA == P_DBL_CPLX || modeA == P_DBL_SPLIT) return 1;
  if (modeB == P_DBL_CPLX || modeB == P_DBL_SPLIT) return 2;
  return 0;
}

// C' = A' B'^T over packed operands; the epilogue writes FP64/FP32 C (c != null)
// or the next stage's packed operand (po != null)
template <int ESZ>
static cudaError_t launch_split(const SplitPacked& A, const SplitPacked& B, int M, int N, int batch,
                                const GemmParams* c, const SplitPackOut* po, cudaStream_t st) {
  CUtensorMap tAh, tAl, tBh, tBl;
  if (A.kext != B.kext) return cudaErrorInvalidValue;
  if (!make_map(&tAh, A.hi, ESZ, A.kext, A.pitch, A.rows, A.nb, BM) ||
      !make_map(&tAl, A.lo, ESZ, A.kext, A.pitch, A.rows, A.nb, BM) ||
      !make_map(&tBh, B.hi, ESZ, B.kext, B.pitch, B.rows, B.nb, BN) ||
      !make_map(&tBl, B.lo, ESZ, B.kext, B.pitch, B.rows, B.nb, BN))
    return cudaErrorInvalidValue;
  const int inter = inter_of(A.mode, B.mode);
  Epi epi{};
  epi.M = M;
  epi.N = N;
  epi.rows_p = (int)A.rows;
  epi.cols_p = (int)B.rows;
  if (po) {
    epi.mode = OUT_PACK;
    epi.phi = po->hi;
    epi.plo = po->lo;
    epi.s_b = po->s_b;
    epi.s_m1 = po->s_m1;
    epi.s_m0 = po->s_m0;
    epi.s_n1 = po->s_n1;
    epi.s_n0 = po->s_n0;
    epi.s_ri = po->s_ri;
    epi.Dm = po->Dm > 0 ? po->Dm : 1 << 30;
    epi.Dn = po->Dn > 0 ? po->Dn : 1 << 30;
    epi.inter = inter;
  } else {
    epi.mode = inter == 1 ? OUT_ROWS_CPLX : inter == 2 ? OUT_COLS_CPLX : OUT_REAL;
    epi.C = c->C;
    epi.sCm = c->sCm;
    epi.sCn = c->sCn;
    epi.sCb = c->sCb;
    epi.accumulate = c->accumulate;
    epi.c_f32 = c->c_f32;
  }
  const int64_t kstep = KROW_BYTES / ESZ;
  const int chunk_k = g_split_chunk_k.load(std::memory_order_relaxed);
  const int kc = chunk_k > 0 ? (int)std::max<int64_t>(1, chunk_k / kstep) : 0;
  static std::atomic<unsigned long long> smem_set{0}, smem_set_p{0};
  {
    cudaError_t e = kc > 0 ? smem_optin_once(split_gemm_kernel<ESZ, true>, SMEM_BYTES, smem_set_p)
                           : smem_optin_once(split_gemm_kernel<ESZ, false>, SMEM_BYTES, smem_set);
    if (e != cudaSuccess) return e;
  }
  const int64_t mt = ceil_div(A.rows, BM), nt = ceil_div(B.rows, BN);
  // walk the smaller operand's tiles fastest (packed rows per batch decide)
  const int m_fast = (A.rows <= B.rows && mt > 1) ? 1 : 0;
  const int64_t ntiles = mt * nt * (int64_t)batch;
  if (ntiles > 0x7fffffff) return cudaErrorInvalidValue;
  const int sms = sm_count_current_device();
  const int grid = (int)std::min<int64_t>(ntiles, sms);  // one persistent CTA per SM
  count_launch();
  const uint64_t wait_ns = g_wait_ns.load(std::memory_order_relaxed);
  const int skip = g_skip_split_stage.exchange(-1);
  const int nkt = (int)ceil_div(A.kext, kstep);
  if (kc > 0)
    split_gemm_kernel<ESZ, true><<<grid, THREADS, SMEM_BYTES, st>>>(
        tAh, tAl, tBh, tBl, epi, nkt, (int)A.kext, A.nb > 1 ? 1 : 0, B.nb > 1 ? 1 : 0, m_fast, (int)mt, (int)nt,
        (int)ntiles, wait_ns, skip, kc);
  else
    split_gemm_kernel<ESZ, false><<<grid, THREADS, SMEM_BYTES, st>>>(
        tAh, tAl, tBh, tBl, epi, nkt, (int)A.kext, A.nb > 1 ? 1 : 0, B.nb > 1 ? 1 : 0, m_fast, (int)mt, (int)nt,
        (int)ntiles, wait_ns, skip, 0);
  return cudaGetLastError();
}

template <int ESZ>
static cudaError_t run_split(const GemmParams& p, const Plan& q, char* ws, cudaStream_t st) {
  SplitPacked A{ws + q.offAh, ws + q.offAl, q.pitch, q.rowsA, q.nbA, q.KA, q.modeA};
  SplitPacked B{ws + q.offBh, ws + q.offBl, q.pitch, q.rowsB, q.nbB, q.KA, q.modeB};
  cudaError_t e = run_pack<ESZ>(p.A, p.M, p.K, (int)q.nbA, q.modeA, SplitRows{}, A.hi, A.lo, q.pitch, q.rowsA, st);
  if (e == cudaSuccess) e = run_pack<ESZ>(p.B, p.N, p.K, (int)q.nbB, q.modeB, SplitRows{}, B.hi, B.lo, q.pitch, q.rowsB, st);
  if (e != cudaSuccess) return e;
  return launch_split<ESZ>(A, B, p.M, p.N, p.batch, &p, nullptr, st);
}

}  // namespace split

size_t split_gemm_required_bytes(const GemmParams& p, int prec) {
  if (prec == RENO_PREC_FP64 || p.M <= 0 || p.N <= 0 || p.batch <= 0) return 0;
  return split::make_plan(p, prec).total;
}

size_t split_gemm_workspace_bytes(int64_t a_elems, int64_t b_elems) {
  // conservative: complex operands doubled and K-concatenated, hi+lo, 4-byte elements
  return (size_t)(8 * 4 * 2) * (size_t)(a_elems + b_elems) + (size_t)(64 << 20);
}

cudaError_t split_gemm(const GemmParams& p, int prec, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return cudaSuccess;
  if (p.K <= 0) return (p.A.is_f32 || p.B.is_f32 || p.c_f32) ? cudaErrorInvalidValue : gemm_fp64(p, st);
  const split::Plan q = split::make_plan(p, prec);
  if (q.total > ws_bytes || !ws) return cudaErrorInvalidValue;
  if (q.esz == 2) return split::run_split<2>(p, q, static_cast<char*>(ws), st);
  return split::run_split<4>(p, q, static_cast<char*>(ws), st);
}

int split_esz(int prec) { return prec == RENO_PREC_BF16X3 ? 2 : 4; }

int64_t split_pitch(int64_t kext, int prec) {
  const int64_t align = 16 / split_esz(prec);
  return ((kext + align - 1) / align) * align;
}

size_t split_packed_bytes(int64_t rows, int64_t kext, int64_t nb, int prec) {
  return 2 * split::al((size_t)rows * split_pitch(kext, prec) * nb * split_esz(prec));
}

SplitPacked split_packed_at(void* base, int64_t rows, int64_t kext, int64_t nb, int mode, int prec) {
  const size_t plane = split::al((size_t)rows * split_pitch(kext, prec) * nb * split_esz(prec));
  return SplitPacked{base, static_cast<char*>(base) + plane, split_pitch(kext, prec), rows, nb, kext, mode};
}

cudaError_t split_pack(const GemmOperand& op, int R, int K, int nb, const SplitRows& rs, const SplitPacked& dst,
                       int prec, cudaStream_t st) {
  if (R <= 0 || K <= 0 || nb <= 0) return cudaSuccess;
  if (split_esz(prec) == 2)
    return split::run_pack<2>(op, R, K, nb, dst.mode, rs, dst.hi, dst.lo, dst.pitch, dst.rows, st);
  return split::run_pack<4>(op, R, K, nb, dst.mode, rs, dst.hi, dst.lo, dst.pitch, dst.rows, st);
}

cudaError_t split_run(const SplitPacked& A, const SplitPacked& B, int M, int N, int batch, const GemmParams* c,
                      const SplitPackOut* po, int prec, cudaStream_t st) {
  if (M <= 0 || N <= 0 || batch <= 0) return cudaSuccess;
  if ((c == nullptr) == (po == nullptr)) return cudaErrorInvalidValue;
  if (split_esz(prec) == 2) return split::launch_split<2>(A, B, M, N, batch, c, po, st);
  return split::launch_split<4>(A, B, M, N, batch, c, po, st);
}

int split_gemm_take_error() {
  int h = 0;
  cudaMemcpyFromSymbol(&h, split::g_split_error, sizeof(int));
  if (h) {
    int z = 0;
    cudaMemcpyToSymbol(split::g_split_error, &z, sizeof(int));
  }
  return h;
}

}  // namespace reno
