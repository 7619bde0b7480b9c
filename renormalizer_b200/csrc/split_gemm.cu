// Split-precision complex GEMM on the 5th-generation tensor cores (sm_100a).
//
// C (FP64, real or complex) = opA(A) opB(B) with A, B FP64 (real or complex,
// any strides), computed as
//     A ~ A_hi + A_lo,  B ~ B_hi + B_lo    (BF16 or TF32 pairs)
//     C ~ A_hi B_hi + A_hi B_lo + A_lo B_hi   (FP32 accumulation in TMEM)
// Complex operands use the real embedding: the smaller operand is "doubled"
// into [[Re, -Im], [Im, Re]] rows, the other is K-concatenated as [Re | Im],
// so each complex GEMM is ONE real GEMM whose rows (or columns) interleave the
// real and imaginary parts of the result.
//
// Pipeline (one 128 x 256 output tile per CTA, 6 warps):
//   warp 0     TMA producer: 4 tiles per stage (A_hi, A_lo, B_hi, B_lo),
//              128-byte swizzled K-major boxes, mbarrier complete_tx
//   warp 1     TMEM allocator + single-thread tcgen05.mma issuer: 3 products
//              per stage, tcgen05.commit frees the stage
//   warps 2-5  epilogue: tcgen05.ld 32x32b from TMEM, FP32 -> FP64, strided
//              writes of the (interleaved complex) output
// Every mbarrier wait is bounded; on timeout the kernel records the site in
// a device error word, skips the remaining work and still frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstring>
#include "split_gemm.cuh"

namespace reno {
namespace split {

constexpr int BM = 128, BN = 256, STAGES = 2, THREADS = 192;
constexpr int KROW_BYTES = 128;  // one SW128 row of K per stage
constexpr int A_TILE = BM * KROW_BYTES;   // 16 KB
constexpr int B_TILE = BN * KROW_BYTES;   // 32 KB
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr uint32_t TMEM_COLS = 256;
constexpr uint64_t WAIT_NS = 2000000000ull;  // bounded spin: 2 s of wall clock

// device error word: 0 = ok; otherwise 1000 + site of the first timed-out wait
__device__ int g_split_error = 0;

enum OutMode { OUT_REAL = 0, OUT_COLS_CPLX = 1, OUT_ROWS_CPLX = 2 };

struct Epi {
  void* C;
  int64_t sCm, sCn, sCb;  // output strides in output elements
  int M, N;               // logical output dims
  int mode;
  int accumulate;
  int rows_p, cols_p;     // rows / cols of the real product C' actually present
};

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

// bounded wait (WAIT_NS of wall clock): returns false and raises the abort flag on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int site) {
  const uint64_t t0 = global_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255u) == 255u) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > WAIT_NS) break;
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

template <int ESZ>
__global__ void __launch_bounds__(THREADS, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                      const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl, Epi epi,
                      int num_k_tiles, int a_batched, int b_batched, int m_fast) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* tmem_full = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tmem_full + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // m_fast: consecutive CTAs walk the M tiles of one N tile, so a large B
  // operand streams from HBM once while the small A operand stays in L2
  const int m_tile = m_fast ? blockIdx.x : blockIdx.y, n_tile = m_fast ? blockIdx.y : blockIdx.x, bz = blockIdx.z;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tmem_full, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    const int za = a_batched ? bz : 0, zb = b_batched ? bz : 0;
    for (int kt = 0; kt < num_k_tiles; ++kt) {
      const int s = kt % STAGES;
      const uint32_t ph = (kt / STAGES) & 1;
      if (!mbar_wait(&empty[s], ph ^ 1, abort_flag, 1)) break;
      unsigned char* st = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      const int kx = kt * (KROW_BYTES / ESZ);
      tma_load_3d(st, &tmAh, &full[s], kx, m_tile * BM, za);
      tma_load_3d(st + A_TILE, &tmAl, &full[s], kx, m_tile * BM, za);
      tma_load_3d(st + 2 * A_TILE, &tmBh, &full[s], kx, n_tile * BN, zb);
      tma_load_3d(st + 2 * A_TILE + B_TILE, &tmBl, &full[s], kx, n_tile * BN, zb);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    constexpr uint32_t fmt = ESZ == 2 ? 1u : 2u;  // BF16 : TF32
    const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    bool ok = true;
    for (int kt = 0; kt < num_k_tiles && ok; ++kt) {
      const int s = kt % STAGES;
      const uint32_t ph = (kt / STAGES) & 1;
      if (!mbar_wait(&full[s], ph, abort_flag, 2)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
      const uint64_t dah = sdesc(base), dal = sdesc(base + A_TILE);
      const uint64_t dbh = sdesc(base + 2 * A_TILE), dbl = sdesc(base + 2 * A_TILE + B_TILE);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint64_t adv = (uint64_t)((kk * 32) >> 4);  // 32 bytes of K per instruction
        const uint32_t first = (kt == 0 && kk == 0) ? 0u : 1u;
        umma<ESZ>(tmem, dah + adv, dbh + adv, idesc, first);
        umma<ESZ>(tmem, dah + adv, dbl + adv, idesc, 1u);
        umma<ESZ>(tmem, dal + adv, dbh + adv, idesc, 1u);
      }
      umma_commit(&empty[s]);
    }
    umma_commit(tmem_full);
  } else if (warp >= 2) {
    // ---------------- epilogue
    const int q = warp % 4;  // TMEM lane quarter this warp may access
    const bool ok = mbar_wait(tmem_full, 0, abort_flag, 3);
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok && !*abort_flag) {
      const int row = q * 32 + lane;  // tile row of this thread
      const int rp = m_tile * BM + row;
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0;
        TMEM_LD32(taddr, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
        const int cp = n_tile * BN + c0;  // product column of v[0]
        if (epi.mode == OUT_REAL) {
          if (rp < epi.M) {
            double* C = reinterpret_cast<double*>(epi.C) + (int64_t)bz * epi.sCb + (int64_t)rp * epi.sCm;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const int n = cp + j;
              if (n < epi.N) {
                double* p = C + (int64_t)n * epi.sCn;
                *p = (epi.accumulate ? *p : 0.0) + (double)v[j];
              }
            }
          }
        } else if (epi.mode == OUT_COLS_CPLX) {
          if (rp < epi.M) {
            double2* C = reinterpret_cast<double2*>(epi.C) + (int64_t)bz * epi.sCb + (int64_t)rp * epi.sCm;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int n = cp / 2 + j;
              if (n < epi.N) {
                double2* p = C + (int64_t)n * epi.sCn;
                double2 o = epi.accumulate ? *p : make_double2(0.0, 0.0);
                o.x += (double)v[2 * j];
                o.y += (double)v[2 * j + 1];
                *p = o;
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
            double2* C = reinterpret_cast<double2*>(epi.C) + (int64_t)bz * epi.sCb + (int64_t)m * epi.sCm;
            const int nb = cp + (even ? 0 : 16);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int n = nb + j;
              if (n < epi.N) {
                double2* p = C + (int64_t)n * epi.sCn;
                double2 o = epi.accumulate ? *p : make_double2(0.0, 0.0);
                o.x += (double)(even ? mine[j] : got[j]);
                o.y += (double)(even ? got[j] : mine[j]);
                *p = o;
              }
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
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
  int src_complex, conj;
  int64_t s_r, s_k, s_b;  // element strides of rows, K and batch
  int R, K, nbatch, mode;
  void* hi;
  void* lo;
  int64_t pitch;        // K' padded (elements)
  int64_t rows_out;     // rows per batch in the packed buffer
  int64_t kused;        // K' actually written; [kused, pitch) is zeroed
  int kblocks;          // blocks along K that copy data; the block column after them zeroes the padding
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

template <int ESZ>
__device__ __forceinline__ void zero_store(void* hi, void* lo, int64_t idx) {
  if constexpr (ESZ == 2) {
    reinterpret_cast<__nv_bfloat16*>(hi)[idx] = __float2bfloat16(0.f);
    reinterpret_cast<__nv_bfloat16*>(lo)[idx] = __float2bfloat16(0.f);
  } else {
    reinterpret_cast<float*>(hi)[idx] = 0.f;
    reinterpret_cast<float*>(lo)[idx] = 0.f;
  }
}

// one 32 x 32 (rows x K) source tile per block, staged through shared memory so
// that both the strided FP64 reads and the K-contiguous packed writes coalesce;
// the extra block column (blockIdx.x == kblocks) zeroes the K padding
// [kused, pitch) of the packed rows of its 32 source rows
template <int ESZ>
__global__ void pack_kernel(PackArgs a) {
  __shared__ double2 tile[32][33];
  const int b = blockIdx.z;
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  if ((int)blockIdx.x >= a.kblocks) {
    const int64_t base = (int64_t)b * a.rows_out * a.pitch;
    const bool dbl = a.mode == P_DBL_CPLX || a.mode == P_DBL_SPLIT;
    for (int i = ty; i < 32; i += 8) {
      const int r = r0 + i;
      if (r >= a.R) continue;
      for (int rr = 0; rr < (dbl ? 2 : 1); ++rr) {
        const int64_t row = base + (int64_t)(dbl ? 2 * r + rr : r) * a.pitch;
        for (int64_t k = a.kused + tx; k < a.pitch; k += 32) zero_store<ESZ>(a.hi, a.lo, row + k);
      }
    }
    return;
  }
  const bool k_fast = (a.s_k == 1) || (a.s_r != 1);
  for (int i = ty; i < 32; i += 8) {
    const int r = k_fast ? r0 + i : r0 + tx;
    const int k = k_fast ? k0 + tx : k0 + i;
    double2 v = make_double2(0.0, 0.0);
    if (r < a.R && k < a.K) {
      const int64_t off = (int64_t)b * a.s_b + (int64_t)r * a.s_r + (int64_t)k * a.s_k;
      if (a.src_complex) {
        v = reinterpret_cast<const double2*>(a.src)[off];
        if (a.conj) v.y = -v.y;
      } else {
        v.x = reinterpret_cast<const double*>(a.src)[off];
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

static bool make_map(CUtensorMap* tm, void* base, int esz, int64_t pitch, int64_t rows, int64_t nb, int box_rows) {
  EncodeTiledFn enc = encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)rows, (cuuint64_t)nb};
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
  int64_t pitch;         // K' padded to 128-byte rows
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
  q.pitch = ((q.KA + q.kstep - 1) / q.kstep) * q.kstep;
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
static cudaError_t run_pack(const GemmOperand& op, int R, int K, int nb, int mode, void* hi, void* lo, int64_t pitch,
                            int64_t rows_out, int64_t kused, cudaStream_t st) {
  PackArgs a;
  a.src = op.ptr;
  a.src_complex = op.is_complex;
  a.conj = op.conj;
  a.s_r = op.s_outer;
  a.s_k = op.s_k;
  a.s_b = op.s_batch;
  a.R = R;
  a.K = K;
  a.nbatch = nb;
  a.mode = mode;
  a.hi = hi;
  a.lo = lo;
  a.pitch = pitch;
  a.rows_out = rows_out;
  a.kused = kused;
  a.kblocks = (int)ceil_div(K, 32);
  dim3 grid((unsigned)(a.kblocks + (pitch > kused ? 1 : 0)), (unsigned)ceil_div(R, 32), (unsigned)nb);
  count_launch();
  pack_kernel<ESZ><<<grid, dim3(32, 8), 0, st>>>(a);
  return cudaGetLastError();
}

template <int ESZ>
static cudaError_t run_split(const GemmParams& p, const Plan& q, char* ws, cudaStream_t st) {
  void *Ah = ws + q.offAh, *Al = ws + q.offAl, *Bh = ws + q.offBh, *Bl = ws + q.offBl;
  cudaError_t e = run_pack<ESZ>(p.A, p.M, p.K, (int)q.nbA, q.modeA, Ah, Al, q.pitch, q.rowsA, q.KA, st);
  if (e == cudaSuccess) e = run_pack<ESZ>(p.B, p.N, p.K, (int)q.nbB, q.modeB, Bh, Bl, q.pitch, q.rowsB, q.KA, st);
  if (e != cudaSuccess) return e;
  CUtensorMap tAh, tAl, tBh, tBl;
  if (!make_map(&tAh, Ah, ESZ, q.pitch, q.rowsA, q.nbA, BM) || !make_map(&tAl, Al, ESZ, q.pitch, q.rowsA, q.nbA, BM) ||
      !make_map(&tBh, Bh, ESZ, q.pitch, q.rowsB, q.nbB, BN) || !make_map(&tBl, Bl, ESZ, q.pitch, q.rowsB, q.nbB, BN))
    return cudaErrorInvalidValue;
  Epi epi;
  epi.C = p.C;
  epi.sCm = p.sCm;
  epi.sCn = p.sCn;
  epi.sCb = p.sCb;
  epi.M = p.M;
  epi.N = p.N;
  epi.mode = q.out;
  epi.accumulate = p.accumulate;
  epi.rows_p = (int)q.rowsA;
  epi.cols_p = (int)q.rowsB;
  static bool attr_set = false;
  if (!attr_set) {
    e = cudaFuncSetAttribute(split_gemm_kernel<ESZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int64_t mt = ceil_div(q.rowsA, BM), nt = ceil_div(q.rowsB, BN);
  // walk the smaller operand's tiles fastest (packed rows per batch decide)
  const int m_fast = (q.rowsA <= q.rowsB && mt > 1 && nt <= 65535) ? 1 : 0;
  dim3 grid((unsigned)(m_fast ? mt : nt), (unsigned)(m_fast ? nt : mt), (unsigned)p.batch);
  count_launch();
  split_gemm_kernel<ESZ><<<grid, THREADS, SMEM_BYTES, st>>>(tAh, tAl, tBh, tBl, epi, (int)(q.pitch / q.kstep),
                                                            q.nbA > 1 ? 1 : 0, q.nbB > 1 ? 1 : 0, m_fast);
  return cudaGetLastError();
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
  if (p.K <= 0) return gemm_fp64(p, st);
  const split::Plan q = split::make_plan(p, prec);
  if (q.total > ws_bytes || !ws) return cudaErrorInvalidValue;
  if (q.esz == 2) return split::run_split<2>(p, q, static_cast<char*>(ws), st);
  return split::run_split<4>(p, q, static_cast<char*>(ws), st);
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
