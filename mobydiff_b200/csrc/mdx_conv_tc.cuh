// mdx_conv_tc.cuh -- 3x3x3 convolution of the learned warm start on the
// Blackwell tensor cores (tcgen05.mma, FP32 accumulators in tensor memory).
//
// Implicit GEMM: D[128 voxels x COUT] += A[128 x 16] B[16 x COUT] for every
// tap (27) and 16-channel slice of the input, for RY output rows of 128
// consecutive x voxels (one accumulator of COUT tensor-memory columns per
// row).  Activations are channels-last BF16 [z][y][x][C]; input planes --
// 130 x voxels (x0-1 .. x0+128) by RY+2 rows, wrapped in x and z (and y when
// periodic), zero beyond y walls -- are staged in shared memory as
// [y][8-channel chunk][x][8 x bf16], so that the A
// operand of a tap is the same canonical no-swizzle K-major layout shifted
// by whole 16-byte voxels: core matrices of 8 voxels x 16 bytes, 128 bytes
// apart along M, one halo row apart (130 x 16 bytes) along K.  The weights
// [tap][cout][cin] are staged as [tap][chunk][cout][8 x bf16].  One thread
// issues the MMAs, tcgen05.commit arrives on an mbarrier when they are done,
// and the four warps read their 32 tensor-memory lanes (voxels) back with
// tcgen05.ld for the epilogue (bias + leaky ReLU to BF16, or FP32 as is).
//
// Needs the level's nx to be a multiple of 128 (whole tiles in x); other
// levels keep the mma.sync kernel.  Every A descriptor reads 128 voxels
// starting at halo voxel 0, 1 or 2 of a staged row, and the next 8-channel
// chunk of the same row: inside the halo by construction.
#pragma once

#include <cuda_bf16.h>

namespace tc {

constexpr int XT = 128;            // voxels per output row (the MMA's M)
constexpr int HXT = XT + 2;        // halo voxels per row
constexpr int THREADS = 128;       // one warpgroup: four warps own the 128 tensor-memory lanes
constexpr unsigned long long WAIT_NS = 1000000000ull;

__device__ __forceinline__ unsigned s32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, canonical layout without swizzle.
__device__ __forceinline__ unsigned long long sdesc(unsigned addr, unsigned lbo, unsigned sbo) {
    unsigned long long d = 0;
    d |= (unsigned long long)((addr & 0x3FFFFu) >> 4);
    d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;   // descriptor version of this architecture
    return d;          // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr unsigned idesc_bf16(int m, int n) {
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((unsigned)(n >> 3) << 17)   // N / 8
           | ((unsigned)(m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(unsigned dtmem, unsigned long long a, unsigned long long b, unsigned idesc,
                                         unsigned accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ bool bar_try(unsigned bar, unsigned phase) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(phase)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned phase) {
    if (bar_try(bar, phase)) return true;
    const unsigned long long t0 = gtime();
    while (!bar_try(bar, phase))
        if (gtime() - t0 > WAIT_NS) return false;
    return true;
}

template <int N>
__device__ __forceinline__ void tmem_ld(unsigned taddr, float* v);
template <>
__device__ __forceinline__ void tmem_ld<16>(unsigned taddr, float* v) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
template <>
__device__ __forceinline__ void tmem_ld<32>(unsigned taddr, float* v) {
    tmem_ld<16>(taddr, v);
    tmem_ld<16>(taddr + 16, v + 16);
}

}  // namespace tc

// ---------------------------------------------------------------------------
// The staging is pipelined across z: a CTA walks a chunk of zc planes for one
// (128-voxel x, RY-row y) column.  Its weights are staged once; input planes
// sit in a ring of 4 slots (plane z in slot (z - z_first + 1) mod 4); each
// step issues the MMAs of plane z into one of two accumulator sets, then --
// while they run -- reads back the other set (plane z-1) for the epilogue
// and, once plane z-1's MMAs are done, stages plane z+2 into the slot plane
// z-2 used.  EPI 0: y = leaky(acc + bias) stored BF16; EPI 1: acc stored FP32.
// Grid: (nx/128) x ceil(ny/RY) x ceil(nz/zc).  *err is set when a bounded
// wait gives up.
// ---------------------------------------------------------------------------
namespace tc {
template <int CIN, int COUT, int RY>
struct pgeom {
    static constexpr int CH = CIN / 8;
    static constexpr int SLOTS = 4;
    static constexpr int PLANE_BYTES = (RY + 2) * CH * HXT * 16;
    static constexpr int W_BYTES = 27 * CH * COUT * 16;
    static constexpr int NCOL = 2 * RY * COUT;   // two accumulator sets
    static constexpr int COLS = NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : (NCOL <= 256 ? 256 : 512)));
    static constexpr int SMEM = 128 + W_BYTES + SLOTS * PLANE_BYTES;
};
}  // namespace tc

template <int CIN, int COUT, int EPI, int RY, typename LVL>
__global__ void __launch_bounds__(tc::THREADS, 1)
k_conv3_tcp(LVL L, int pery, int zc, const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ W,
            const float* __restrict__ bias, float slope, __nv_bfloat16* __restrict__ Yb, float* __restrict__ Yf,
            int* __restrict__ err) {
    using G = tc::pgeom<CIN, COUT, RY>;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);   // two mbarriers
    unsigned* taddr_slot = reinterpret_cast<unsigned*>(smem + 16);
    unsigned char* sw = smem + 128;
    unsigned char* ring = sw + G::W_BYTES;
    const int x0 = blockIdx.x * tc::XT, y0 = blockIdx.y * RY, zb = blockIdx.z * zc;
    const int nsteps = min(zc, L.nz - zb);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc::s32(taddr_slot)),
                     "r"((unsigned)G::COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc::s32(bars)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc::s32(bars + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    for (int q = threadIdx.x; q < 27 * COUT * G::CH; q += tc::THREADS) {
        const int ch = q % G::CH, row = q / G::CH;
        const int tap = row / COUT, co = row - tap * COUT;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::s32(sw + ((tap * G::CH + ch) * COUT + co) * 16)),
                     "l"(W + (long long)row * CIN + ch * 8));
    }
    auto slot_of = [&](int z) { return (z - zb + 1) & (G::SLOTS - 1); };
    auto stage = [&](int z) {   // plane z (wrapped) into its slot
        int gz = z < 0 ? z + L.nz : (z >= L.nz ? z - L.nz : z);
        unsigned char* base = ring + slot_of(z) * G::PLANE_BYTES;
        for (int q = threadIdx.x; q < (RY + 2) * G::CH * tc::HXT; q += tc::THREADS) {
            const int hx = q % tc::HXT;
            const int rest = q / tc::HXT;
            const int ch = rest % G::CH, hy = rest / G::CH;
            int gx = x0 + hx - 1, gy = y0 + hy - 1;
            gx = gx < 0 ? gx + L.nx : (gx >= L.nx ? gx - L.nx : gx);
            bool ok = true;
            if (pery) gy = gy < 0 ? gy + L.ny : (gy >= L.ny ? gy - L.ny : gy);
            else ok = gy >= 0 && gy < L.ny;
            unsigned char* dst = base + ((hy * G::CH + ch) * tc::HXT + hx) * 16;
            if (ok)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::s32(dst)),
                             "l"(X + ((((long long)gz * L.ny + gy) * L.nx + gx) * CIN + ch * 8)));
            else
                *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
        }
    };
    stage(zb - 1);
    stage(zb);
    if (nsteps > 0) stage(zb + 1);
    asm volatile("cp.async.commit_group;\n" ::);

    unsigned tmem = 0;
    auto epilogue = [&](int q) {   // plane zb+q from accumulator set q & 1
        const int z = zb + q;
        const int x = x0 + warp * 32 + lane;
        for (int r = 0; r < RY; ++r) {
            float v[COUT];
            tc::tmem_ld<COUT>(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(((q & 1) * RY + r) * COUT), v);
            const int y = y0 + r;
            if (y >= L.ny) continue;
            const long long vox = ((long long)z * L.ny + y) * L.nx + x;
            if (EPI == 0) {
                __align__(16) __nv_bfloat16 o[COUT];
#pragma unroll
                for (int c = 0; c < COUT; ++c) {
                    float t = v[c] + bias[c];
                    t = t > 0.f ? t : t * slope;
                    o[c] = __float2bfloat16_rn(t);
                }
#pragma unroll
                for (int c = 0; c < COUT; c += 8)
                    *reinterpret_cast<uint4*>(Yb + vox * COUT + c) = *reinterpret_cast<const uint4*>(o + c);
            } else {
#pragma unroll
                for (int c = 0; c < COUT; c += 4)
                    *reinterpret_cast<float4*>(Yf + vox * COUT + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
            }
        }
    };

    bool ok = true;
    for (int q = 0; q < nsteps; ++q) {
        const int z = zb + q;
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");   // planes z-1 .. z+1 (and the weights) staged
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        tmem = *taddr_slot;
        if (threadIdx.x == 0) {
            // Descriptors differ only in their start address (bits 0-13, in 16-byte
            // units, all addresses below 256 KB): build each once and add offsets
            // that are compile-time constants but for the three plane slots.
            constexpr unsigned idesc = tc::idesc_bf16(128, COUT);
            const unsigned long long b0 = tc::sdesc(tc::s32(sw), COUT * 16, 128);
            const unsigned long long a0 = tc::sdesc(tc::s32(ring), tc::HXT * 16, 128);
            const unsigned long long as[3] = {a0 + (unsigned)(slot_of(z - 1) * G::PLANE_BYTES / 16),
                                              a0 + (unsigned)(slot_of(z) * G::PLANE_BYTES / 16),
                                              a0 + (unsigned)(slot_of(z + 1) * G::PLANE_BYTES / 16)};
            const unsigned dset = tmem + (unsigned)((q & 1) * RY * COUT);
#pragma unroll
            for (int r = 0; r < RY; ++r)
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
#pragma unroll
                    for (int kc = 0; kc < CIN / 16; ++kc) {
                        const unsigned aoff = ((r + dy + 1) * G::CH + 2 * kc) * tc::HXT + (dx + 1);
                        const unsigned boff = (tap * G::CH + 2 * kc) * COUT;
                        tc::mma_bf16(dset + (unsigned)(r * COUT), as[dz + 1] + aoff, b0 + boff, idesc,
                                     (tap | kc) != 0);
                    }
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             tc::s32(bars + (q & 1)))
                         : "memory");
        }
        if (q > 0) {   // plane z-1: its MMAs done, then its epilogue; its slot z-2 is free afterwards
            const bool done = tc::bar_wait(tc::s32(bars + ((q - 1) & 1)), (unsigned)(((q - 1) >> 1) & 1));
            if (__syncthreads_or(!done)) { ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue(q - 1);
        }
        if (q + 1 < nsteps) stage(z + 2);
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    if (ok && nsteps > 0) {
        const int q = nsteps - 1;
        const bool done = tc::bar_wait(tc::s32(bars + (q & 1)), (unsigned)((q >> 1) & 1));
        if (__syncthreads_or(!done)) ok = false;
        else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue(q);
        }
    }
    if (!ok) {   // a wait gave up: flag it and give the MMAs in flight one more bounded wait
        if (threadIdx.x == 0) atomicExch(err, 1);
        tc::bar_wait(tc::s32(bars), 0);
        tc::bar_wait(tc::s32(bars + 1), 0);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem ? tmem : *taddr_slot),
                     "r"((unsigned)G::COLS)
                     : "memory");
}
