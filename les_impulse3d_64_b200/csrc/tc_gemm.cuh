// tc_gemm.cuh - the FDM transforms of the mixed form on the 5th-generation tensor cores (tcgen05), FP32-accurate
// through the 3xTF32 split: every fp32 operand x is written as hi + lo with hi = x rounded to TF32 and lo = x - hi,
// and a product is accumulated as a_lo b_hi + a_hi b_lo + a_hi b_hi in FP32 (the a_lo b_lo term is below fp32
// rounding).  This is the mixed form's counterpart of the reference's FP32 SGEMM transforms (backend.cu:792-814);
// the FP64 form keeps its FP64 DMMA transforms (fdm.cuh).
//
// One launch computes C[b] (M x N) = A[b] (M x K) * B[b] (K x N) for one of the six transforms of a pass.
// One operand is the field (fp32 t1/t2, or the fp64 residual scaled by 1/rms in the first transform) and the
// other a basis S or S^T of one axis, pre-split at set-up into hi/lo "images" laid out in shared-memory order.
//
//  * field_is_a = 1 (the x transforms): A = field rows [m][k], B = basis image.
//  * field_is_a = 0 (the y and z transforms): A = basis image, B = field [k][n] (n contiguous), transposed into
//    the K-major layout on its way to shared memory.
//
// Both operands sit in shared memory in the K-major, non-swizzled canonical layout.  A CTA of 128 threads owns a
// 128 x BN tile of C held in TMEM (128 lanes x BN fp32 columns).  K runs in panels of 32 through two
// shared-memory stages: the threads load panel p+1 (field values split into hi/lo, one 16-byte shared store per
// 4 consecutive k; cp.async copies of the basis image) while the tensor core works on panel p.  One
// thread issues the tcgen05.mma.cta_group::1.kind::tf32 instructions (M = 128, N = BN, K = 8) and commits each
// panel to that stage's mbarrier.  Every mbarrier wait is bounded: on time-out the kernel records
// kDeviceWait in the control block, frees its TMEM and returns.  Only this kernel and the staged one below
// allocate TMEM, and their shared memory (>= 80 KB; 192 KB for the staged kernel's 128 columns) keeps at most two
// CTAs of <= 64 columns, or one of 128, on an SM, below its 512 columns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "kernels.cuh"

namespace cavity {

constexpr int kTcThreads = 128;
constexpr int kTcKC = 32;                 // K panel
constexpr int kTcRows = 128;              // M of the tile (TMEM lanes)

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle: start address, LBO = byte distance between core matrices adjacent
// along K, SBO = between core matrices adjacent along M/N, version 1 (sm_100), layout type 0 (no swizzle)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// instruction descriptor of kind::tf32 with fp32 accumulation; a_mn / b_mn = 1 would select MN-major operands
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase of parity `parity` of an mbarrier to complete; false on time-out (~0.3 s)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (long it = 0; it < (1L << 22); it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t* result, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(result)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}
__device__ __forceinline__ void cp_async16_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void st_shared4(uint32_t addr, float a, float b, float c, float d) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}

// ---------------------------------------------------------------- 3xTF32 split
// hi = x rounded to the nearest TF32 value (10 explicit mantissa bits), lo = x - hi (exact in fp32).  Inf and NaN
// pass through hi so that a blown-up field still shows in the residual.
__host__ __device__ inline void tf32_split(float x, float& hi, float& lo) {
    uint32_t bits;
    memcpy(&bits, &x, 4);
    if ((bits & 0x7F800000u) == 0x7F800000u) { hi = x; lo = 0.0f; return; }
    const uint32_t hb = (bits + 0x1000u) & 0xFFFFE000u;
    memcpy(&hi, &hb, 4);
    lo = x - hi;
}

// ---------------------------------------------------------------- layouts
// K-major, no swizzle: core matrices of 8 rows x 16 bytes (4 elements along K); K-adjacent cores 128 bytes apart
// (LBO), 8-row groups kTcKC/4 * 128 = 1024 bytes apart (SBO).  Byte offset of (row r, k) in a 32-wide K panel:
__host__ __device__ constexpr int kmajor_off(int r, int k) {
    return ((r >> 3) * (kTcKC / 4) + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4;
}
constexpr uint32_t kKmajorLBO = 128, kKmajorSBO = (kTcKC / 4) * 128;

// A basis image holds the hi (or lo) parts of a matrix with `rows` rows and k columns, rows rounded up to 128 (R)
// and columns to 32, zero-padded, panel by panel: panel p is the K-major shared-memory image of rows 0..R-1 and
// columns 32p..32p+31, so that rows [r0, r0 + n) of panel p are the n * 128 contiguous bytes from byte
// (p * R + r0) * 128.  Element (r, k) is at float (k / 32) * R * 32 + kmajor_off(r, k % 32) / 4.
__host__ __device__ constexpr int basis_image_rows(int rows) { return (rows + kTcRows - 1) / kTcRows * kTcRows; }
__host__ __device__ constexpr long long basis_image_floats(int rows, int k) {
    return (long long)basis_image_rows(rows) * ((k + kTcKC - 1) / kTcKC * kTcKC);
}
__host__ __device__ constexpr long long basis_image_index(int R, int r, int k) {
    return (long long)(k / kTcKC) * R * kTcKC + kmajor_off(r, k % kTcKC) / 4;
}

enum TcEpilogue : int { kTcStore = 0, kTcScaleInvLambda = 1, kTcAccumulate = 2 };

struct TcTransformArgs {
    int M, N, K;                   // per batch entry
    int field_is_a;
    const float* field;            // fp32 field, or
    const double* field64;         // fp64 field scaled by 1/rms on load (first transform of a pass)
    const double* field64_alt;     // replaces field64 when the control block says use_rhs
    long long field_bstride;       // batch stride of the field (elements)
    int field_ld;                  // row pitch of the field (elements)
    const float* basis_hi;         // images (see basis_image_floats)
    const float* basis_lo;
    int basis_rows;                // R of the images
    float* out;
    long long out_bstride;
    int out_ld;
    const float* inv_lambda;       // kTcScaleInvLambda: indexed like out
    double* phi;                   // kTcAccumulate: phi[i] = (reset ? 0 : phi[i]) + rms * C (indexed like out)
    int epilogue;
    double n_cell;                 // rms = sqrt(|r|^2 / n_cell)
    const Control* c;
    int* error;                    // where a timed-out wait is recorded (the control block's error word)
    cudaGraphConditionalHandle handle;
    int clear_condition;
};

template <int BN> struct TcSmem {
    static constexpr int kA = kTcRows * kTcKC * 4;      // bytes of one A panel part (hi or lo)
    static constexpr int kB = BN * kTcKC * 4;
    static constexpr int kStage = 2 * kA + 2 * kB;
    static constexpr int kBytes = 2 * kStage;
};

// Work item e of an A panel (128 rows x 8 groups of 4 k): the 8 lanes of a quarter-warp take 8 consecutive rows at
// one k group, so that their 16-byte shared stores fill one 128-byte row of core matrices without bank conflicts,
// and a warp's 4 quarters take 4 consecutive k groups, so that it reads 64 contiguous bytes of each of its rows.
__device__ __forceinline__ void fa_item(int e, int& r, int& k4) {
    const int hi = e >> 5;
    r = (e & 7) + 8 * (hi >> 1);
    k4 = ((e >> 3) & 3) + 4 * (hi & 1);
}

// The field side of a K panel in registers: FA (field is A) = 128 rows x 32 k, float4 (or two double2 when the
// source is the fp64 residual) per 4 consecutive k; otherwise 32 k x BN n, as (n, 4 consecutive k) quadruples.
template <int BN, int FA, int F64> struct FieldPanel {
    static constexpr int kSlots = FA ? kTcRows * kTcKC / 4 / kTcThreads : BN * kTcKC / 4 / kTcThreads;
    float4 v[F64 ? 1 : kSlots];
    double2 d[F64 ? 2 * kSlots : 1];
};

// grid: (N / BN tiles, M / 128 tiles, batch).  FA: the field is operand A (x transforms); F64: the field is the
// fp64 residual, scaled by 1/rms (first transform of a pass).
template <int BN, int FA, int F64>
__device__ void tc_transform_body(const TcTransformArgs& g, const Blk& blk, bool first) {
    using L = TcSmem<BN>;
    using P = FieldPanel<BN, FA, F64>;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const int b = blk.z;
    const int m0 = blk.y * kTcRows, n0 = blk.x * BN;
    const int row = m0 + warp * 32 + lane;
    const uint32_t sbase = smem_addr(smem);
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;
    // TMEM and the barriers are set up while the previous kernel finishes (programmatic dependent launch); at
    // most two CTAs of this kernel and two of a preceding one share an SM, within its 512 TMEM columns
    pdl_launch_dependents();
    if (warp == 0) tmem_alloc(&tmem_base, kCols);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        failed = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    pdl_wait();
    if (g.clear_condition && threadIdx.x == 0 && first) cudaGraphSetConditional(g.handle, 0u);
    const Control* c = g.c;
    const int err = c->error, use_rhs = c->use_rhs, reset = c->reset_phi, cond = c->cond;
    const double rhs2 = c->rhs_norm2, res2 = c->res_norm2;
    const double r2 = use_rhs ? rhs2 : res2;
    // failed, this cavity's refinement has ended, or a zero residual: no pass (backend.cu:803-804)
    if (err || !cond || !(r2 > 0)) {
        if (warp == 0) tmem_dealloc(tmem, kCols);
        return;
    }
    const double rms = sqrt(r2 / g.n_cell);
    const double inv_rms = 1.0 / rms;
    // the epilogue's other operand (phi or 1/lambda) comes into L2 while the panels are multiplied
    if (row < g.M && g.epilogue != kTcStore && !(g.epilogue == kTcAccumulate && reset)) {
        const long long base = b * g.out_bstride + (long long)row * g.out_ld + n0;
        const int cnt = min(BN, g.N - n0);
        const char* q = g.epilogue == kTcAccumulate ? (const char*)(g.phi + base) : (const char*)(g.inv_lambda + base);
        const int bytes = cnt * (g.epilogue == kTcAccumulate ? 8 : 4);
        for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(q + o));
    }
    const float* F = F64 ? nullptr : g.field + b * g.field_bstride;
    const double* Fd = F64 ? ((use_rhs && g.field64_alt) ? g.field64_alt : g.field64) + b * g.field_bstride : nullptr;
    const int panels = (g.K + kTcKC - 1) / kTcKC;

    // issue the field loads of panel p (values stay in flight until store_field uses them)
    auto load_field = [&](P& f, int p) {
        const int k0 = p * kTcKC;
#pragma unroll
        for (int j = 0; j < P::kSlots; j++) {
            const int e = tid + j * kTcThreads;
            if (FA) {                                          // (row, 4 consecutive k): see fa_item
                int r, k4;
                fa_item(e, r, k4);
                const int k = k0 + k4 * 4, gm = m0 + r;
                const bool ok = gm < g.M && k < g.K;
                const long long gi = (long long)gm * g.field_ld + k;
                if (F64) {
                    f.d[2 * j] = ok ? *reinterpret_cast<const double2*>(Fd + gi) : make_double2(0.0, 0.0);
                    f.d[2 * j + 1] = ok ? *reinterpret_cast<const double2*>(Fd + gi + 2) : make_double2(0.0, 0.0);
                } else {
                    f.v[j] = ok ? *reinterpret_cast<const float4*>(F + gi) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            } else {                                           // (n, 4 consecutive k); a warp reads 32 n of a row
                const int n = e % BN, k = k0 + (e / BN) * 4, gn = n0 + n;
                const float* src = F + (long long)k * g.field_ld + gn;
                const long long ld = g.field_ld;
                const bool okn = gn < g.N;
                f.v[j] = make_float4(okn && k < g.K ? src[0] : 0.f, okn && k + 1 < g.K ? src[ld] : 0.f,
                                     okn && k + 2 < g.K ? src[2 * ld] : 0.f, okn && k + 3 < g.K ? src[3 * ld] : 0.f);
            }
        }
    };
    // split panel values into hi/lo and store them in the K-major layout of stage s
    auto store_field = [&](const P& f, int s) {
        const uint32_t st = sbase + s * L::kStage + (FA ? 0 : 2 * L::kA);
        const uint32_t part = FA ? L::kA : L::kB;
#pragma unroll
        for (int j = 0; j < P::kSlots; j++) {
            const int e = tid + j * kTcThreads;
            float4 x;
            if (F64)
                x = make_float4((float)(f.d[2 * j].x * inv_rms), (float)(f.d[2 * j].y * inv_rms),
                                (float)(f.d[2 * j + 1].x * inv_rms), (float)(f.d[2 * j + 1].y * inv_rms));
            else
                x = f.v[F64 ? 0 : j];
            int r, k4;
            if (FA) fa_item(e, r, k4);
            else { r = e % BN; k4 = e / BN; }
            const uint32_t off = kmajor_off(r, k4 * 4);
            float h0, l0, h1, l1, h2, l2, h3, l3;
            tf32_split(x.x, h0, l0);
            tf32_split(x.y, h1, l1);
            tf32_split(x.z, h2, l2);
            tf32_split(x.w, h3, l3);
            st_shared4(st + off, h0, h1, h2, h3);
            st_shared4(st + part + off, l0, l1, l2, l3);
        }
    };
    // the basis side of panel p into stage s: rows [row0, row0 + rows) of the images, contiguous bytes
    auto copy_basis = [&](int p, int s) {
        const uint32_t st = sbase + s * L::kStage;
        constexpr int rows = FA ? BN : kTcRows;
        const int row0 = FA ? n0 : m0;
        const uint32_t dst = FA ? st + 2 * L::kA : st;
        constexpr uint32_t part = FA ? L::kB : L::kA;
        const long long src = ((long long)p * g.basis_rows + row0) * kTcKC;      // floats
        constexpr int chunks = rows * kTcKC / 4;                                  // 16-byte pieces per part
#pragma unroll
        for (int e = tid; e < chunks; e += kTcThreads) {
            cp_async16(dst + e * 16, g.basis_hi + src + e * 4);
            cp_async16(dst + part + e * 16, g.basis_lo + src + e * 4);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    const uint32_t idesc = umma_idesc_tf32(kTcRows, BN, 0, 0);
    // panel p: the loads of panel p+1 go out first and stay in flight while panel p (loaded one step earlier
    // into `cur`) is split, stored and multiplied.  Two register sets alternate (the loop is unrolled by two),
    // so no register copy ever waits on a load.  Returns false when a bounded wait ran out.
    auto panel = [&](int p, const P& cur, P& next) -> bool {
        const int s = p & 1;
        if (p + 1 < panels) load_field(next, p + 1);
        store_field(cur, s);                                  // stage s is free: MMA(p-2) finished before basis(p)
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // basis(p) has landed
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t st = sbase + s * L::kStage;
            const uint32_t a_hi = st, a_lo = st + L::kA, b_hi = st + 2 * L::kA, b_lo = b_hi + L::kB;
#pragma unroll
            for (int ks = 0; ks < kTcKC / 8; ks++) {                         // 8 k = two core matrices = 256 B
                const uint64_t ah = umma_desc(a_hi + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t al = umma_desc(a_lo + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t bh = umma_desc(b_hi + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t bl = umma_desc(b_lo + ks * 256, kKmajorLBO, kKmajorSBO);
                umma_tf32(tmem, al, bh, idesc, (p > 0 || ks > 0) ? 1u : 0u);
                umma_tf32(tmem, ah, bl, idesc, 1u);
                umma_tf32(tmem, ah, bh, idesc, 1u);
            }
            umma_commit(&mbar[s]);
        }
        if (p + 1 < panels) {
            // stage s^1 was read by MMA(p-1): wait for it, then bring in the basis of panel p+1
            if (p >= 1 && !mbar_wait_bounded(&mbar[s ^ 1], ((p - 1) >> 1) & 1)) failed = 1;
            __syncthreads();
            if (failed) return false;
            copy_basis(p + 1, s ^ 1);
        }
        return true;
    };
    P fa, fb;
    load_field(fa, 0);
    copy_basis(0, 0);
    for (int p = 0; p < panels; p += 2) {
        if (!panel(p, fa, fb)) break;
        if (p + 1 < panels && !panel(p + 1, fb, fa)) break;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (!failed && !mbar_wait_bounded(&mbar[(panels - 1) & 1], ((panels - 1) >> 1) & 1)) failed = 1;
    tc_fence_after();
    __syncthreads();
    if (failed) {
        if (tid == 0) atomicExch(g.error, (int)kDeviceWait);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(tmem, kCols);
        return;
    }
    // epilogue through shared memory (free once every MMA has completed): warp w moves TMEM lanes (tile rows)
    // 32w..32w+31 into a row-major tile with a pitch of BN + 4 floats (conflict-free 16-byte writes), then
    // writes its rows back with BN/4 lanes per row, so that every warp access covers contiguous columns.
    constexpr int kPitch = BN + 4;
    static_assert(kTcRows * kPitch * 4 <= L::kBytes, "epilogue tile exceeds the stages");
    float* tile = reinterpret_cast<float*>(smem) + warp * 32 * kPitch;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
        float* dst = tile + lane * kPitch + c0;
#pragma unroll
        for (int q = 0; q < 4; q++)
            *reinterpret_cast<float4*>(dst + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
    __syncwarp();
    constexpr int kLanesPerRow = BN / 4, kRowsPerStep = 32 / kLanesPerRow;
    const int lr = lane / kLanesPerRow, lc = (lane % kLanesPerRow) * 4;
    const int gcol = n0 + lc;
#pragma unroll 4
    for (int r0 = 0; r0 < 32; r0 += kRowsPerStep) {
        const int rl = r0 + lr, grow = m0 + warp * 32 + rl;
        if (grow >= g.M || gcol >= g.N) continue;             // N is a multiple of 4: a float4 is all in or out
        float4 x = *reinterpret_cast<const float4*>(tile + rl * kPitch + lc);
        const long long idx = b * g.out_bstride + (long long)grow * g.out_ld + gcol;
        if (g.epilogue == kTcAccumulate) {
            double2 p0 = make_double2(0.0, 0.0), p1 = make_double2(0.0, 0.0);
            if (!reset) {
                p0 = *reinterpret_cast<const double2*>(g.phi + idx);
                p1 = *reinterpret_cast<const double2*>(g.phi + idx + 2);
            }
            p0.x += (double)x.x * rms; p0.y += (double)x.y * rms;
            p1.x += (double)x.z * rms; p1.y += (double)x.w * rms;
            *reinterpret_cast<double2*>(g.phi + idx) = p0;
            *reinterpret_cast<double2*>(g.phi + idx + 2) = p1;
        } else {
            if (g.epilogue == kTcScaleInvLambda) {
                const float4 il = *reinterpret_cast<const float4*>(g.inv_lambda + idx);
                x.x *= il.x; x.y *= il.y; x.z *= il.z; x.w *= il.w;
            }
            *reinterpret_cast<float4*>(g.out + idx) = x;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
}

template <int BN, int FA, int F64>
__global__ void __launch_bounds__(kTcThreads) tc_transform_kernel(TcTransformArgs g) {
    tc_transform_body<BN, FA, F64>(g, real_blk(), first_block());
}
// a batch of cavities: grid x runs over the work list (BatchItem)
template <int BN, int FA, int F64>
__global__ void __launch_bounds__(kTcThreads) tc_transform_batched(const TcTransformArgs* args, const BatchItem* items,
                                                                   const int* live) {
    __shared__ TcTransformArgs g;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) {
        dead_slot_clear(args, items);
        return;
    }
    load_args(g, args + cav);
    tc_transform_body<BN, FA, F64>(g, k, first_block());
}

// ---------------------------------------------------------------- staged kernel
// The same transform with the field brought in like the basis: every copy of a K panel (basis image and raw
// field) is a cp.async issued NS - 1 panels ahead into a ring of NS shared-memory stages, and the field is split
// into hi/lo in place once its panel has landed, so the K loop waits for no load.  256 threads share the copies
// and the split; each thread's copy and split addresses are fixed for the whole K loop (only a panel offset
// moves), so a panel costs a few instructions per element.  A CTA owns a 128 x BN tile.
//  * field is A (x transforms): the raw fp32 values of 4 consecutive k of a row are one 16-byte copy into the
//    hi image; the fp64 residual's (first transform) are two, into the hi and the lo image, scaled by 1/rms and
//    rounded to float by the split;
//  * field is B (y, z transforms: [k][n], n contiguous): one 4-byte copy per element into its K-major place, the
//    lanes of a warp taking consecutive n of one k row.
constexpr int kTc2Threads = 256;
template <int BN, int NS> struct Tc2Smem {
    static constexpr int kA = kTcRows * kTcKC * 4;      // bytes of one A panel part (hi or lo)
    static constexpr int kB = BN * kTcKC * 4;
    static constexpr int kStage = 2 * kA + 2 * kB;
    static constexpr int kBytes = NS * kStage;
};
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async16s(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ float4 ld_shared4(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
    return v;
}
__device__ __forceinline__ double2 ld_shared2d(uint32_t addr) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(addr));
    return v;
}
// cp.async.wait_group with a run-time count of at most two groups still in flight
__device__ __forceinline__ void cp_async_wait_le(int n) {
    if (n <= 0) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    else if (n == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else asm volatile("cp.async.wait_group 2;\n" ::: "memory");
}
// byte offset of k within a 32-wide K panel's core-matrix rows (kmajor_off(r, k) - kmajor_off(r, 0))
__host__ __device__ constexpr int kmajor_koff(int k) { return (k >> 2) * 128 + (k & 3) * 4; }

template <int BN, int NS, int FA, int F64>
__device__ void tc2_transform_body(const TcTransformArgs& g, const Blk& blk, bool first) {
    static_assert(NS >= 2 && NS <= 3, "cp_async_wait_le covers at most two outstanding panels");
    constexpr int NT = kTc2Threads;
    static_assert(NT == 256 && (BN == 64 || BN == 128), "copy plans below assume 256 threads");
    using L = Tc2Smem<BN, NS>;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[NS];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const int b = blk.z;
    const int m0 = blk.y * kTcRows, n0 = blk.x * BN;
    const uint32_t sbase = smem_addr(smem);
    pdl_launch_dependents();
    if (warp == 0) tmem_alloc(&tmem_base, BN);
    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&mbar[s], 1);
        failed = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    pdl_wait();
    if (g.clear_condition && threadIdx.x == 0 && first) cudaGraphSetConditional(g.handle, 0u);
    const Control* c = g.c;
    const int err = c->error, use_rhs = c->use_rhs, reset = c->reset_phi, cond = c->cond;
    const double rhs2 = c->rhs_norm2, res2 = c->res_norm2;
    const double r2 = use_rhs ? rhs2 : res2;
    if (err || !cond || !(r2 > 0)) {                       // no pass (backend.cu:803-804)
        if (warp == 0) tmem_dealloc(tmem, BN);
        return;
    }
    const double rms = sqrt(r2 / g.n_cell);
    const double inv_rms = 1.0 / rms;
    const float* F = F64 ? nullptr : g.field + b * g.field_bstride;
    const double* Fd = F64 ? ((use_rhs && g.field64_alt) ? g.field64_alt : g.field64) + b * g.field_bstride : nullptr;
    const int panels = (g.K + kTcKC - 1) / kTcKC;
    const long long ld = g.field_ld;

    // ---- copy plan, fixed over the K loop
    // basis: rows [row0, row0 + BR) of a panel's images are BR * 128 contiguous bytes, 16 per copy
    constexpr int BR = FA ? BN : kTcRows, BQ = BR * 8 / NT;
    constexpr uint32_t kBasisDst = FA ? 2 * L::kA : 0, kBasisPart = FA ? L::kB : L::kA;
    const long long bsrc0 = (long long)(FA ? n0 : m0) * kTcKC + tid * 4;       // floats, panel 0
    const long long bstep = (long long)g.basis_rows * kTcKC;
    // field as A: thread t copies rows r_t + 32 q (q < 4) at the 4 k of group k4_t (fa_item of t + 256 q)
    const int fr_t = (tid & 7) + 8 * (warp >> 1), fk4_t = ((tid >> 3) & 3) + 4 * (warp & 1);
    const uint32_t fa_off = kmajor_off(fr_t, 4 * fk4_t);
    // field as B: thread t copies n = t % BN at k = h + S q (h = t / BN, S = 256 / BN)
    constexpr int S = NT / BN, BQN = BN * kTcKC / NT;
    const int bn_t = tid % BN, bh_t = tid / BN;
    const uint32_t fb_off = 2 * L::kA + kmajor_off(bn_t, 0) + 4 * bh_t;
    const bool fb_ok = n0 + bn_t < g.N;

    auto issue = [&](int p, int s) {
        const uint32_t st = sbase + s * L::kStage;
        const int k0 = p * kTcKC;
        const long long bsrc = bsrc0 + p * bstep;
#pragma unroll
        for (int q = 0; q < BQ; q++) {
            cp_async16(st + kBasisDst + (tid + q * NT) * 16, g.basis_hi + bsrc + q * NT * 4);
            cp_async16(st + kBasisDst + kBasisPart + (tid + q * NT) * 16, g.basis_lo + bsrc + q * NT * 4);
        }
        if (FA) {
            const int k = k0 + 4 * fk4_t;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int gm = m0 + fr_t + 32 * q;
                const bool ok = gm < g.M && k < g.K;
                const uint32_t off = st + fa_off + q * 4096;
                if (F64) {
                    const double* src = Fd + gm * ld + k;
                    cp_async16s(off, ok ? src : Fd, ok ? 16 : 0);
                    cp_async16s(off + L::kA, ok ? src + 2 : Fd, ok ? 16 : 0);
                } else {
                    cp_async16s(off, ok ? F + gm * ld + k : F, ok ? 16 : 0);
                }
            }
        } else {
            const float* src = F + (long long)(k0 + bh_t) * ld + n0 + bn_t;
#pragma unroll
            for (int q = 0; q < BQN; q++) {
                const bool ok = fb_ok && k0 + bh_t + S * q < g.K;
                cp_async4(st + fb_off + kmajor_koff(S * q), ok ? src + S * q * ld : F, ok ? 4 : 0);
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    // split the landed field of stage s in place: hi image <- TF32(x), lo image <- x - hi
    auto split = [&](int s) {
        const uint32_t st = sbase + s * L::kStage;
        constexpr uint32_t part = FA ? L::kA : L::kB;
#pragma unroll
        for (int q = 0; q < (FA ? 4 : BN * 8 / NT); q++) {
            const uint32_t off = FA ? st + fa_off + q * 4096
                                    : st + 2 * L::kA + kmajor_off(bn_t, 0) + (bh_t + S * q) * 128;
            float4 x;
            if (F64) {
                const double2 d01 = ld_shared2d(off), d23 = ld_shared2d(off + part);     // k, k+1 and k+2, k+3
                x = make_float4((float)(d01.x * inv_rms), (float)(d01.y * inv_rms), (float)(d23.x * inv_rms),
                                (float)(d23.y * inv_rms));
            } else {
                x = ld_shared4(off);
            }
            float h0, l0, h1, l1, h2, l2, h3, l3;
            tf32_split(x.x, h0, l0);
            tf32_split(x.y, h1, l1);
            tf32_split(x.z, h2, l2);
            tf32_split(x.w, h3, l3);
            st_shared4(off, h0, h1, h2, h3);
            st_shared4(off + part, l0, l1, l2, l3);
        }
    };

    // the epilogue's other operand (phi or 1/lambda) comes into L2 while the panels are multiplied
    {
        const int row = m0 + (tid & 127), half = tid >> 7;
        if (row < g.M && g.epilogue != kTcStore && !(g.epilogue == kTcAccumulate && reset)) {
            const int c0 = n0 + half * (BN / 2);
            const long long base = b * g.out_bstride + (long long)row * g.out_ld + c0;
            const int cnt = min(BN / 2, g.N - c0);
            const int esz = g.epilogue == kTcAccumulate ? 8 : 4;
            const char* q = g.epilogue == kTcAccumulate ? (const char*)(g.phi + base) : (const char*)(g.inv_lambda + base);
            for (int o = 0; o < cnt * esz; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(q + o));
        }
    }
    const uint32_t idesc = umma_idesc_tf32(kTcRows, BN, 0, 0);
    int issued = 0;
    for (; issued < panels && issued < NS; issued++) issue(issued, issued);
    for (int p = 0; p < panels; p++) {
        const int s = p % NS;
        cp_async_wait_le(issued - p - 1);                  // this thread's copies of panel p have landed
        __syncthreads();                                    // ... and every thread's
        split(s);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t st = sbase + s * L::kStage;
            const uint32_t a_hi = st, a_lo = st + L::kA, b_hi = st + 2 * L::kA, b_lo = b_hi + L::kB;
#pragma unroll
            for (int ks = 0; ks < kTcKC / 8; ks++) {
                const uint64_t ah = umma_desc(a_hi + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t al = umma_desc(a_lo + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t bh = umma_desc(b_hi + ks * 256, kKmajorLBO, kKmajorSBO);
                const uint64_t bl = umma_desc(b_lo + ks * 256, kKmajorLBO, kKmajorSBO);
                umma_tf32(tmem, al, bh, idesc, (p > 0 || ks > 0) ? 1u : 0u);
                umma_tf32(tmem, ah, bl, idesc, 1u);
                umma_tf32(tmem, ah, bh, idesc, 1u);
            }
            umma_commit(&mbar[s]);
        }
        // the stage of panel p - 1 is free once its MMAs are done: it takes the next panel
        if (p >= 1 && issued < panels) {
            const int q = p - 1;
            if (!mbar_wait_bounded(&mbar[q % NS], (q / NS) & 1)) failed = 1;
            __syncthreads();
            if (failed) break;
            issue(issued, issued % NS);
            issued++;
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (!failed && !mbar_wait_bounded(&mbar[(panels - 1) % NS], ((panels - 1) / NS) & 1)) failed = 1;
    tc_fence_after();
    __syncthreads();
    if (failed) {
        if (tid == 0) atomicExch(g.error, (int)kDeviceWait);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(tmem, BN);
        return;
    }
    // epilogue through shared memory: warp w moves TMEM lanes 32 (w % 4) .. + 31, columns of half w / 4, into a
    // row-major tile (pitch BN + 4 floats); then every warp writes 16 whole rows back, row-contiguous
    constexpr int kPitch = BN + 4;
    static_assert(kTcRows * kPitch * 4 <= L::kBytes, "epilogue tile exceeds the stages");
    float* tile = reinterpret_cast<float*>(smem);
    {
        const int lb = warp & 3, half = warp >> 2;
#pragma unroll 1
        for (int c0 = half * (BN / 2); c0 < (half + 1) * (BN / 2); c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(lb * 32) << 16) + c0, v);
            float* dst = tile + (lb * 32 + lane) * kPitch + c0;
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<float4*>(dst + 4 * q) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
    }
    __syncthreads();
    constexpr int kLanesPerRow = BN / 4, kRowsPerStep = 32 / kLanesPerRow;
    const int lr = lane / kLanesPerRow, lc = (lane % kLanesPerRow) * 4;
    const int gcol = n0 + lc;
#pragma unroll 2
    for (int r0 = 0; r0 < kTcRows / 8; r0 += kRowsPerStep) {
        const int rl = warp * (kTcRows / 8) + r0 + lr, grow = m0 + rl;
        if (grow >= g.M || gcol >= g.N) continue;          // N is a multiple of 4: a float4 is all in or out
        float4 x = *reinterpret_cast<const float4*>(tile + rl * kPitch + lc);
        const long long idx = b * g.out_bstride + (long long)grow * g.out_ld + gcol;
        if (g.epilogue == kTcAccumulate) {
            double2 p0 = make_double2(0.0, 0.0), p1 = make_double2(0.0, 0.0);
            if (!reset) {
                p0 = *reinterpret_cast<const double2*>(g.phi + idx);
                p1 = *reinterpret_cast<const double2*>(g.phi + idx + 2);
            }
            p0.x += (double)x.x * rms; p0.y += (double)x.y * rms;
            p1.x += (double)x.z * rms; p1.y += (double)x.w * rms;
            *reinterpret_cast<double2*>(g.phi + idx) = p0;
            *reinterpret_cast<double2*>(g.phi + idx + 2) = p1;
        } else {
            if (g.epilogue == kTcScaleInvLambda) {
                const float4 il = *reinterpret_cast<const float4*>(g.inv_lambda + idx);
                x.x *= il.x; x.y *= il.y; x.z *= il.z; x.w *= il.w;
            }
            *reinterpret_cast<float4*>(g.out + idx) = x;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, BN);
}

// tile width and ring depth of the staged kernel (compile-time; -DCAVITY_TC2_BN / -DCAVITY_TC2_NS override)
#ifndef CAVITY_TC2_BN
#define CAVITY_TC2_BN 128
#endif
#ifndef CAVITY_TC2_NS
#define CAVITY_TC2_NS 3
#endif
constexpr int kTc2BN = CAVITY_TC2_BN, kTc2NS = CAVITY_TC2_NS;
constexpr int kTcStagedVariant = 1 << 10;      // flag of a recorded launch of the staged kernel
template <int FA, int F64>
__global__ void __launch_bounds__(kTc2Threads) tc2_transform_kernel(TcTransformArgs g) {
    tc2_transform_body<kTc2BN, kTc2NS, FA, F64>(g, real_blk(), first_block());
}
template <int FA, int F64>
__global__ void __launch_bounds__(kTc2Threads) tc2_transform_batched(const TcTransformArgs* args, const BatchItem* items,
                                                                     const int* live) {
    __shared__ TcTransformArgs g;
    int cav;
    const Blk k = item_blk(items, live, cav);
    if (cav < 0) {
        dead_slot_clear(args, items);
        return;
    }
    load_args(g, args + cav);
    tc2_transform_body<kTc2BN, kTc2NS, FA, F64>(g, k, first_block());
}

// ---------------------------------------------------------------- host side
// tile width: 64 columns when that still gives one CTA per SM, else 32.  (128-column tiles would need 128 KB of
// shared memory, one CTA per SM, and each CTA's K loop is latency-bound: two CTAs per SM of 64 columns are faster.)
inline int tc_pick_bn(int M, int N, int batch, int sms) {
    const long long mt = (M + kTcRows - 1) / kTcRows;
    return (long long)((N + 63) / 64) * mt * batch >= sms ? 64 : 32;
}
// once per device, before any capture: the dynamic shared memory of every instance
template <int BN> inline cudaError_t tc_prepare_bn() {
    cudaError_t e = cudaFuncSetAttribute(tc_transform_kernel<BN, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TcSmem<BN>::kBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_transform_kernel<BN, 1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcSmem<BN>::kBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_transform_kernel<BN, 0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcSmem<BN>::kBytes);
    return e;
}
template <int BN> inline cudaError_t tc_prepare_batched_bn() {
    cudaError_t e = cudaFuncSetAttribute(tc_transform_batched<BN, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TcSmem<BN>::kBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_transform_batched<BN, 1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcSmem<BN>::kBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_transform_batched<BN, 0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcSmem<BN>::kBytes);
    return e;
}
inline cudaError_t tc2_prepare() {
    constexpr int bytes = Tc2Smem<kTc2BN, kTc2NS>::kBytes;
    cudaError_t e = cudaFuncSetAttribute(tc2_transform_kernel<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tc2_transform_kernel<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tc2_transform_kernel<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tc2_transform_batched<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tc2_transform_batched<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(tc2_transform_batched<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}
inline cudaError_t tc_transform_prepare_batched() {
    cudaError_t e = tc_prepare_batched_bn<64>();
    if (e == cudaSuccess) e = tc_prepare_batched_bn<32>();
    if (e == cudaSuccess) e = tc2_prepare();
    return e;
}
template <int BN>
inline void launch_tc_batched_bn(int fa, int f64, dim3 grid, const BatchItem* items, const int* live,
                                 const TcTransformArgs* d, cudaStream_t st) {
    const dim3 block(kTcThreads);
    if (fa && f64) launch_pdl(tc_transform_batched<BN, 1, 1>, grid, block, TcSmem<BN>::kBytes, st, d, items, live);
    else if (fa) launch_pdl(tc_transform_batched<BN, 1, 0>, grid, block, TcSmem<BN>::kBytes, st, d, items, live);
    else launch_pdl(tc_transform_batched<BN, 0, 0>, grid, block, TcSmem<BN>::kBytes, st, d, items, live);
}
// a recorded launch (variant: see tc_variant) over a batch of cavities
inline void launch_tc_batched(int variant, dim3 grid, const BatchItem* items, const int* live, const TcTransformArgs* d,
                              cudaStream_t st) {
    const int bn = variant & 0xff, fa = (variant >> 8) & 1, f64 = (variant >> 9) & 1;
    if (variant & kTcStagedVariant) {
        constexpr int bytes = Tc2Smem<kTc2BN, kTc2NS>::kBytes;
        const dim3 block(kTc2Threads);
        if (fa && f64) launch_pdl(tc2_transform_batched<1, 1>, grid, block, bytes, st, d, items, live);
        else if (fa) launch_pdl(tc2_transform_batched<1, 0>, grid, block, bytes, st, d, items, live);
        else launch_pdl(tc2_transform_batched<0, 0>, grid, block, bytes, st, d, items, live);
        return;
    }
    if (bn == 64) launch_tc_batched_bn<64>(fa, f64, grid, items, live, d, st);
    else launch_tc_batched_bn<32>(fa, f64, grid, items, live, d, st);
}
inline cudaError_t tc_transform_prepare() {
    cudaError_t e = tc_prepare_bn<64>();
    if (e == cudaSuccess) e = tc_prepare_bn<32>();
    if (e == cudaSuccess) e = tc2_prepare();
    return e;
}
template <int BN> inline void launch_tc_bn(cudaStream_t st, const TcTransformArgs& g, dim3 grid) {
    const dim3 block(kTcThreads);
    if (g.field_is_a && g.field64) launch_pdl(tc_transform_kernel<BN, 1, 1>, grid, block, TcSmem<BN>::kBytes, st, g);
    else if (g.field_is_a) launch_pdl(tc_transform_kernel<BN, 1, 0>, grid, block, TcSmem<BN>::kBytes, st, g);
    else launch_pdl(tc_transform_kernel<BN, 0, 0>, grid, block, TcSmem<BN>::kBytes, st, g);
}
// variant code of a recorded launch: tile width, field-is-A, fp64 field
inline int tc_variant(int bn, const TcTransformArgs& g) { return bn | (g.field_is_a ? 1 << 8 : 0) | (g.field64 ? 1 << 9 : 0); }
// The staged kernel (tc2_transform_body) for a single cavity's launch whose 128 x 128 tiles fit on the SMs at
// once (one CTA per SM): there its deeper prefetch shortens the one CTA chain the launch lasts (C3 pass 84 against
// 88 us).  With more tiles than SMs, and in batches, the register-pipelined kernel, whose two CTAs per SM overlap
// each other's latencies (C6 pass 860 against 872 us).  CAVITY_TC_KERNEL=staged or =panel forces either.
inline bool tc_use_staged(const TcTransformArgs& g, int batch, int sms) {
    static const int forced = [] {
        const char* e = std::getenv("CAVITY_TC_KERNEL");
        if (!e) return -1;
        return std::string(e) == "staged" ? 1 : std::string(e) == "panel" ? 0 : -1;
    }();
    if (forced >= 0) return forced == 1;
    if (g_launch_record) return false;
    const long long tiles = (long long)((g.N + kTc2BN - 1) / kTc2BN) * ((g.M + kTcRows - 1) / kTcRows) * batch;
    return tiles <= sms;
}
inline void launch_tc_transform(cudaStream_t st, const TcTransformArgs& g, int batch, int sms) {
    if (tc_use_staged(g, batch, sms)) {
        const dim3 grid((g.N + kTc2BN - 1) / kTc2BN, (g.M + kTcRows - 1) / kTcRows, batch);
        constexpr int bytes = Tc2Smem<kTc2BN, kTc2NS>::kBytes;
        if (record_launch(kLkTc, tc_variant(kTc2BN, g) | kTcStagedVariant, grid, (size_t)bytes, g)) return;
        const dim3 block(kTc2Threads);
        if (g.field_is_a && g.field64) launch_pdl(tc2_transform_kernel<1, 1>, grid, block, bytes, st, g);
        else if (g.field_is_a) launch_pdl(tc2_transform_kernel<1, 0>, grid, block, bytes, st, g);
        else launch_pdl(tc2_transform_kernel<0, 0>, grid, block, bytes, st, g);
        return;
    }
    const int bn = tc_pick_bn(g.M, g.N, batch * g_launch_batch, sms);
    const dim3 grid((g.N + bn - 1) / bn, (g.M + kTcRows - 1) / kTcRows, batch);
    if (record_launch(kLkTc, tc_variant(bn, g), grid, (size_t)(bn == 64 ? TcSmem<64>::kBytes : TcSmem<32>::kBytes), g))
        return;
    if (bn == 64) launch_tc_bn<64>(st, g, grid);
    else launch_tc_bn<32>(st, g, grid);
}

// hi and lo images of S (transpose = 0: image row r = row r of S) or of S^T (transpose = 1: image row r = column r
// of S) for an n x n row-major double S, rounded to float as the reference keeps S (backend.cu:766-772)
__global__ void basis_image_kernel(const double* S, int n, int transpose, float* hi, float* lo) {
    const int R = basis_image_rows(n), Kp = (n + kTcKC - 1) / kTcKC * kTcKC;
    const long long total = (long long)R * Kp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / Kp), k = (int)(i % Kp);
        const float x = r < n && k < n ? (float)(transpose ? S[(size_t)k * n + r] : S[(size_t)r * n + k]) : 0.0f;
        float h, l;
        tf32_split(x, h, l);
        const long long j = basis_image_index(R, r, k);
        hi[j] = h;
        lo[j] = l;
    }
}
inline void launch_basis_image(cudaStream_t st, const double* S, int n, int transpose, float* hi, float* lo) {
    const long long total = basis_image_floats(n, n);
    basis_image_kernel<<<(unsigned)std::min<long long>((total + 255) / 256, 1024), 256, 0, st>>>(S, n, transpose, hi,
                                                                                                  lo);
}

// the operands of a pass on the tensor cores: per axis the images of S (rows; hi, lo) and of S^T (hi, lo), and
// 1/lambda in float (backend.cu:774-786)
struct TcFdmOperands {
    int nx, ny, nz;
    const float* img[3][4];
    const float* inv_lambda;
};

// One pass of backend.cu:801-814 on the tensor cores: r (or r_alt when the control block says use_rhs) scaled
// to rms 1 in the x transform's loads; t = S_z^T S_y^T (r S_x) in fp32 through t1/t2 (nx*ny*nz floats each);
// t *= 1/lambda; phi += rms * (S_z S_y t) S_x^T in the last transform's epilogue.  `clear` makes the first launch
// clear the condition of the enclosing graph while-node `h`.  Needs nx % 4 == 0 (float4 row loads).
inline void launch_tc_fdm_pass(cudaStream_t st, const TcFdmOperands& op, const double* r, const double* r_alt,
                               double* phi, float* t1, float* t2, Control* c, cudaGraphConditionalHandle h, bool clear,
                               int sms) {
    const int nx = op.nx, ny = op.ny, nz = op.nz, plane = nx * ny;
    const int n[3] = {nx, ny, nz};
    TcTransformArgs g = {};
    g.n_cell = (double)nx * ny * nz;
    g.c = c;
    g.error = &c->error;
    g.inv_lambda = op.inv_lambda;
    g.phi = phi;
    g.handle = h;
    auto basis = [&](int a, bool transpose) {
        g.basis_hi = op.img[a][transpose ? 2 : 0];
        g.basis_lo = op.img[a][transpose ? 3 : 1];
        g.basis_rows = basis_image_rows(n[a]);
    };
    // x: rows of the field are the ny*nz x-lines; forward t1 = r S_x, inverse phi += rms * t1 S_x^T
    auto x_transform = [&](const float* f, bool inverse) {
        g.M = ny * nz; g.N = nx; g.K = nx; g.field_is_a = 1;
        g.field = f; g.field64 = inverse ? nullptr : r; g.field64_alt = inverse ? nullptr : r_alt;
        g.field_bstride = 0; g.field_ld = nx;
        basis(0, !inverse);
        g.out = t1; g.out_bstride = 0; g.out_ld = nx;
        g.epilogue = inverse ? kTcAccumulate : kTcStore;
        launch_tc_transform(st, g, 1, sms);
    };
    // y (each z layer) and z: out = S^T in (forward) or S in (inverse)
    auto yz_transform = [&](int a, const float* in, float* out, bool inverse, int epi) {
        const bool y = a == 1;
        g.M = y ? ny : nz; g.N = y ? nx : plane; g.K = g.M; g.field_is_a = 0;
        g.field = in; g.field64 = nullptr; g.field64_alt = nullptr;
        g.field_bstride = y ? plane : 0; g.field_ld = y ? nx : plane;
        basis(a, !inverse);
        g.out = out; g.out_bstride = y ? plane : 0; g.out_ld = y ? nx : plane;
        g.epilogue = epi;
        launch_tc_transform(st, g, y ? nz : 1, sms);
    };
    g.clear_condition = clear;
    x_transform(nullptr, false);
    g.clear_condition = 0;
    yz_transform(1, t1, t2, false, kTcStore);
    yz_transform(2, t2, t1, false, kTcScaleInvLambda);
    yz_transform(2, t1, t2, true, kTcStore);
    yz_transform(1, t2, t1, true, kTcStore);
    x_transform(t1, true);
}

// the squared norm of r into the control block of a standalone pass (one block, fixed order)
__global__ void __launch_bounds__(kThreads) control_norm_kernel(const double* r, long long n, Control* c) {
    Vec<1> acc;
    acc.v[0] = 0.0;
    for (long long i = threadIdx.x; i < n; i += kThreads) acc.v[0] += r[i] * r[i];
    const Vec<1> tot = block_reduce<1, false>(acc);
    if (threadIdx.x == 0) {
        c->res_norm2 = tot.v[0];
        c->rhs_norm2 = tot.v[0];
    }
}

}  // namespace cavity
