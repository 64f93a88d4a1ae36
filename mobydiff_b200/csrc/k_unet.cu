// k_unet.cu -- learned warm start of the red-black projection: a 4-level 3-D
// U-Net trained on the device on snapshots the projection records.
//
// Network (channels c0 at full resolution, c1 at the three coarser levels):
//   enc0a 16->c0, enc0b c0->c0 = s0          level 0 (input: 4 of 16 channels used)
//   pool; enc1a c0->c1, enc1b c1->c1 = s1    level 1
//   pool; enc2a c1->c1, enc2b c1->c1 = s2    level 2
//   pool; enc3a, enc3b (+ extra) c1->c1 = b  level 3
//   dec2 = conv(up(b) + s2)   c1->c1         level 2
//   dec1 = conv(up(dec2) + s1) c1->c0        level 1
//   dec0 = conv(up(dec1) + s0) c0->c0        level 0
//   out  = 1x1 head c0->1 (FP32)
// Every 3x3x3 convolution is followed by a leaky ReLU; pool is the mean of
// 2x2x2 cells, up repeats a cell 2x2x2.  Boundaries: periodic in x and z,
// zero padding at y walls (periodic when y is).
//
// Layout: activations channels-last BF16 [z][y][x][c], c in {16, 32}, on
// the unpadded cells of each level.  Weights BF16 [tap][cout][cin] for the
// forward pass and [26-tap][cin][cout] for the data gradient; FP32 master
// weights, gradients and Adam moments in one flat vector.
//
// Kernels: on levels whose nx is a multiple of 128 the forward convolution
// and the data gradient run on the tcgen05 tensor cores with accumulators in
// tensor memory (k_conv3_tcp, mdx_conv_tc.cuh); elsewhere, and for the weight
// gradient, the 3x3x3 convolution is an implicit GEMM on mma.sync
// m16n8k16 (BF16 in, FP32 accumulate).  A CTA computes a 16x4x4 tile of
// output cells times all output channels: its input halo (18x6x6 cells) and
// all 27 taps of the weights are staged in shared memory by cp.async, and
// the A (cells x input channels of one tap) and B fragments are read with
// ldmatrix from rows whose 16-byte chunks are XOR-swizzled so that eight
// consecutive cells hit eight distinct bank groups.  The data gradient is
// the same kernel on the transposed, flipped weights with an FP32 output.
// The weight gradient is a persistent kernel: each CTA accumulates
// dW[tap][cout][cin] over its tiles in registers (A = gradient tile read
// transposed, B = shifted input halo read transposed) and writes one partial
// per CTA; a column sum reduces them in a fixed order.
#include "mdx_internal.cuh"

#include <cuda_bf16.h>

#include "mdx_conv_tc.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

typedef __nv_bfloat16 bf16;

namespace {

constexpr int TX = 16, TY = 4, TZ = 4;   // output tile of the convolutions
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HV = HX * HY * HZ;         // cells of the input halo
constexpr int TV = TX * TY * TZ;         // cells of the tile (256)
constexpr int NIN = 5;                   // input channels used
constexpr int C_IN = 16;                 // input channels stored (zero padded)
constexpr int MAX_EXTRA = 8;

struct lvl {
    int nx, ny, nz;
    long long n;
};

__device__ __forceinline__ int wrapi(int a, int n) {
    a %= n;
    return a < 0 ? a + n : a;
}

// Byte offset of 16-byte chunk `chunk` of row `row` holding C bf16 values.
template <int C>
__host__ __device__ __forceinline__ int sw_off(int row, int chunk) {
    const int s = (C == 32) ? ((row >> 1) & 3) : ((row >> 2) & 1);
    return row * (C * 2) + ((chunk ^ s) << 4);
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp16(void* s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(s)), "l"(g));
}
__device__ __forceinline__ void cp_commit_wait() {
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ void ldsm4(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm4t(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ int tiles_of(const lvl& L) {
    return ((L.nx + TX - 1) / TX) * ((L.ny + TY - 1) / TY) * ((L.nz + TZ - 1) / TZ);
}
__device__ __forceinline__ void tile_origin(const lvl& L, int b, int& x0, int& y0, int& z0) {
    const int tx = (L.nx + TX - 1) / TX, ty = (L.ny + TY - 1) / TY;
    x0 = (b % tx) * TX;
    y0 = ((b / tx) % ty) * TY;
    z0 = (b / (tx * ty)) * TZ;
}

// Input halo of the tile at (x0,y0,z0): cells x0-1..x0+16, y0-1..y0+4,
// z0-1..z0+4, wrapped in x and z (and y when periodic), zero beyond walls.
template <int C, int NTH>
__device__ __forceinline__ void stage_halo(unsigned char* sx, const bf16* __restrict__ X, const lvl& L, int pery,
                                           int x0, int y0, int z0) {
    constexpr int CH = C / 8;
    for (int q = threadIdx.x; q < HV * CH; q += NTH) {
        const int hv = q / CH, ch = q - hv * CH;
        const int hx = hv % HX, hy = (hv / HX) % HY, hz = hv / (HX * HY);
        const int gx = wrapi(x0 + hx - 1, L.nx), gz = wrapi(z0 + hz - 1, L.nz);
        int gy = y0 + hy - 1;
        bool ok = true;
        if (pery) gy = wrapi(gy, L.ny);
        else ok = gy >= 0 && gy < L.ny;
        unsigned char* dst = sx + sw_off<C>(hv, ch);
        if (ok) cp16(dst, X + ((((long long)gz * L.ny + gy) * L.nx + gx) * C + ch * 8));
        else *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
    }
}

template <int CIN, int COUT>
__host__ __device__ constexpr int conv_smem() {
    return HV * CIN * 2 + 27 * COUT * CIN * 2;
}

// 3x3x3 convolution.  EPI 0: y = leaky(acc + bias) stored BF16; EPI 1: acc
// stored FP32 (data gradient).
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(256) k_conv3(lvl L, int pery, const bf16* __restrict__ X,
                                               const bf16* __restrict__ W, const float* __restrict__ bias,
                                               float slope, bf16* __restrict__ Yb, float* __restrict__ Yf) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sx = smem;
    unsigned char* sw = smem + HV * CIN * 2;
    int x0, y0, z0;
    tile_origin(L, blockIdx.x, x0, y0, z0);
    constexpr int WCH = CIN / 8;
    for (int q = threadIdx.x; q < 27 * COUT * WCH; q += 256) {
        const int row = q / WCH, ch = q - row * WCH;
        cp16(sw + sw_off<CIN>(row, ch), W + (long long)row * CIN + ch * 8);
    }
    stage_halo<CIN, 256>(sx, X, L, pery, x0, y0, z0);
    cp_commit_wait();
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mi = lane >> 3, r8 = lane & 7;
    constexpr int NT = COUT / 8;
    float acc[2][NT][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int n = 0; n < NT; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;

    for (int tap = 0; tap < 27; ++tap) {
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; ++kc) {
            unsigned a[2][4];
#pragma unroll
            for (int m = 0; m < 2; ++m) {
                const int mr = warp * 2 + m;   // x row (ty, tz) of the tile
                const int ty = mr % TY, tz = mr / TY;
                const int hv = (r8 + 8 * (mi & 1) + dx + 1) + HX * ((ty + dy + 1) + HY * (tz + dz + 1));
                ldsm4(a[m], sx + sw_off<CIN>(hv, kc * 2 + (mi >> 1)));
            }
#pragma unroll
            for (int np = 0; np < COUT / 16; ++np) {
                unsigned b[4];
                const int row = tap * COUT + np * 16 + r8 + 8 * (mi >> 1);
                ldsm4(b, sw + sw_off<CIN>(row, kc * 2 + (mi & 1)));
#pragma unroll
                for (int m = 0; m < 2; ++m) {
                    mma16816(acc[m][2 * np], a[m], b[0], b[1]);
                    mma16816(acc[m][2 * np + 1], a[m], b[2], b[3]);
                }
            }
        }
    }

    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        const int mr = warp * 2 + m;
        const int y = y0 + mr % TY, z = z0 + mr / TY;
        if (y >= L.ny || z >= L.nz) continue;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int x = x0 + g + 8 * h;
            if (x >= L.nx) continue;
            const long long v = ((long long)z * L.ny + y) * L.nx + x;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int co = nt * 8 + 2 * t4;
                float v0 = acc[m][nt][2 * h], v1 = acc[m][nt][2 * h + 1];
                if (EPI == 0) {
                    v0 += bias[co];
                    v1 += bias[co + 1];
                    v0 = v0 > 0.f ? v0 : v0 * slope;
                    v1 = v1 > 0.f ? v1 : v1 * slope;
                    *reinterpret_cast<__nv_bfloat162*>(Yb + v * COUT + co) = __floats2bfloat162_rn(v0, v1);
                } else {
                    *reinterpret_cast<float2*>(Yf + v * COUT + co) = make_float2(v0, v1);
                }
            }
        }
    }
}

template <int CIN, int COUT>
__host__ __device__ constexpr int wgrad_warps() {
    return CIN * COUT == 1024 ? 16 : 8;
}
template <int CIN, int COUT>
__host__ __device__ constexpr int wgrad_smem() {
    return HV * CIN * 2 + TV * COUT * 2;
}
template <int CIN, int COUT>
__host__ __device__ constexpr int wgrad_len() {
    return 27 * COUT * CIN + COUT;
}

// Weight and bias gradient of a 3x3x3 convolution: dW[tap][co][ci] =
// sum_v G[v][co] X[v+off(tap)][ci], db[co] = sum_v G[v][co]; one partial per
// CTA in part[blockIdx.x][wgrad_len].
template <int CIN, int COUT>
__global__ void __launch_bounds__(wgrad_warps<CIN, COUT>() * 32, 1)
    k_conv3_wgrad(lvl L, int pery, const bf16* __restrict__ X, const bf16* __restrict__ G, float* __restrict__ part) {
    constexpr int NW = wgrad_warps<CIN, COUT>(), NTH = NW * 32;
    constexpr int MT = COUT / 16, U = 27 * MT, UPW = (U + NW - 1) / NW, NTN = CIN / 8;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sx = smem;
    unsigned char* sg = smem + HV * CIN * 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mi = lane >> 3, r8 = lane & 7;
    float acc[UPW][NTN][4];
#pragma unroll
    for (int u = 0; u < UPW; ++u)
#pragma unroll
        for (int n = 0; n < NTN; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[u][n][e] = 0.f;
    float bsum = 0.f;
    const int ntiles = tiles_of(L);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int x0, y0, z0;
        tile_origin(L, tile, x0, y0, z0);
        __syncthreads();   // the previous tile's reads are done
        stage_halo<CIN, NTH>(sx, X, L, pery, x0, y0, z0);
        constexpr int GCH = COUT / 8;
        for (int q = threadIdx.x; q < TV * GCH; q += NTH) {
            const int v = q / GCH, ch = q - v * GCH;
            const int x = x0 + (v & 15), y = y0 + (v >> 4) % TY, z = z0 + (v >> 4) / TY;
            unsigned char* dst = sg + sw_off<COUT>(v, ch);
            if (x < L.nx && y < L.ny && z < L.nz)
                cp16(dst, G + ((((long long)z * L.ny + y) * L.nx + x) * COUT + ch * 8));
            else
                *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
        }
        cp_commit_wait();
        __syncthreads();
        if (threadIdx.x < COUT) {
            const int co = threadIdx.x;
            for (int v = 0; v < TV; ++v)
                bsum += __bfloat162float(*reinterpret_cast<const bf16*>(sg + sw_off<COUT>(v, co >> 3) + (co & 7) * 2));
        }
        for (int mr = 0; mr < TV / 16; ++mr) {
            const int ty = mr % TY, tz = mr / TY;
#pragma unroll
            for (int u = 0; u < UPW; ++u) {
                const int unit = warp + u * NW;
                if (unit < U) {
                    const int tap = unit / MT, mt = unit - tap * MT;
                    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
                    unsigned a[4];
                    ldsm4t(a, sg + sw_off<COUT>(mr * 16 + r8 + 8 * (mi >> 1), mt * 2 + (mi & 1)));
                    const int hv = (r8 + 8 * (mi & 1) + dx + 1) + HX * ((ty + dy + 1) + HY * (tz + dz + 1));
#pragma unroll
                    for (int np = 0; np < CIN / 16; ++np) {
                        unsigned b[4];
                        ldsm4t(b, sx + sw_off<CIN>(hv, np * 2 + (mi >> 1)));
                        mma16816(acc[u][2 * np], a, b[0], b[1]);
                        mma16816(acc[u][2 * np + 1], a, b[2], b[3]);
                    }
                }
            }
        }
    }
    float* P = part + (long long)blockIdx.x * wgrad_len<CIN, COUT>();
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int u = 0; u < UPW; ++u) {
        const int unit = warp + u * NW;
        if (unit >= U) continue;
        const int tap = unit / MT, mt = unit - tap * MT;
#pragma unroll
        for (int nt = 0; nt < NTN; ++nt) {
            const int ci = nt * 8 + 2 * t4;
            const int co = mt * 16 + g;
            P[((long long)tap * COUT + co) * CIN + ci] = acc[u][nt][0];
            P[((long long)tap * COUT + co) * CIN + ci + 1] = acc[u][nt][1];
            P[((long long)tap * COUT + co + 8) * CIN + ci] = acc[u][nt][2];
            P[((long long)tap * COUT + co + 8) * CIN + ci + 1] = acc[u][nt][3];
        }
    }
    if (threadIdx.x < COUT) P[27 * COUT * CIN + threadIdx.x] = bsum;
}

// out[j] = sum_b part[b][j] in block order.
__global__ void k_sum_parts(int nblk, int len, const float* __restrict__ part, float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= len) return;
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(long long)b * len + j];
    out[j] = s;
}

struct bf8 {
    float v[8];
};
__device__ __forceinline__ bf8 load8(const bf16* p) {
    const uint4 q = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
    bf8 r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        r.v[2 * i] = f.x;
        r.v[2 * i + 1] = f.y;
    }
    return r;
}
__device__ __forceinline__ void store8(bf16* p, const float* v) {
    uint4 q;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4*>(p) = q;
}
__device__ __forceinline__ long long cell_of(const lvl& L, int x, int y, int z) {
    return ((long long)z * L.ny + y) * L.nx + x;
}
__device__ __forceinline__ void coords(const lvl& L, long long v, int& x, int& y, int& z) {
    x = (int)(v % L.nx);
    const long long r = v / L.nx;
    y = (int)(r % L.ny);
    z = (int)(r / L.ny);
}

// Mean of 2x2x2 fine cells -> coarse cell; one thread per (coarse cell, 8 channels).
__global__ void k_pool(lvl Lc, lvl Lf, int C, const bf16* __restrict__ Xf, bf16* __restrict__ Yc) {
    const int CH = C / 8;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < Lc.n * CH;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / CH;
        const int ch = (int)(q - v * CH);
        int x, y, z;
        coords(Lc, v, x, y, z);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = 0; c < 8; ++c) {
            const bf8 a = load8(Xf + cell_of(Lf, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2)) * C + ch * 8);
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += a.v[e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] *= 0.125f;
        store8(Yc + v * C + ch * 8, s);
    }
}

// Y = up(Xc) + S on the fine level.
__global__ void k_up_add(lvl Lf, lvl Lc, int C, const bf16* __restrict__ Xc, const bf16* __restrict__ S,
                         bf16* __restrict__ Y) {
    const int CH = C / 8;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < Lf.n * CH;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / CH;
        const int ch = (int)(q - v * CH);
        int x, y, z;
        coords(Lf, v, x, y, z);
        const bf8 a = load8(Xc + cell_of(Lc, x >> 1, y >> 1, z >> 1) * C + ch * 8);
        const bf8 b = load8(S + v * C + ch * 8);
        float s[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] = a.v[e] + b.v[e];
        store8(Y + v * C + ch * 8, s);
    }
}

// G = bf16((dA + dC[parent]/8) * leaky'(A)) on one level; dA or dC may be null.
__global__ void k_act_bwd_same(lvl L, lvl Lc, int C, const float* __restrict__ dA, const float* __restrict__ dC,
                               const bf16* __restrict__ A, float slope, bf16* __restrict__ G) {
    const int CH = C / 8;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < L.n * CH;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / CH;
        const int ch = (int)(q - v * CH);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (dA) {
            const float4* p = reinterpret_cast<const float4*>(dA + v * C + ch * 8);
            const float4 a = p[0], b = p[1];
            s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
            s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
        }
        if (dC) {
            int x, y, z;
            coords(L, v, x, y, z);
            const float* p = dC + cell_of(Lc, x >> 1, y >> 1, z >> 1) * C + ch * 8;
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += 0.125f * p[e];
        }
        const bf8 a = load8(A + v * C + ch * 8);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] *= a.v[e] > 0.f ? 1.f : slope;
        store8(G + v * C + ch * 8, s);
    }
}

// G = bf16(sum of the 8 fine-cell gradients dF * leaky'(A)) on the coarse level.
__global__ void k_act_bwd_down(lvl Lc, lvl Lf, int C, const float* __restrict__ dF, const bf16* __restrict__ A,
                               float slope, bf16* __restrict__ G) {
    const int CH = C / 8;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < Lc.n * CH;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / CH;
        const int ch = (int)(q - v * CH);
        int x, y, z;
        coords(Lc, v, x, y, z);
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int c = 0; c < 8; ++c) {
            const float* p = dF + cell_of(Lf, 2 * x + (c & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c >> 2)) * C + ch * 8;
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += p[e];
        }
        const bf8 a = load8(A + v * C + ch * 8);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] *= a.v[e] > 0.f ? 1.f : slope;
        store8(G + v * C + ch * 8, s);
    }
}

// Input of the network: in[c][v] (c < NIN) -> X[v][16] BF16.
__global__ void k_pack_in(long long n, const float* __restrict__ in, bf16* __restrict__ X) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int c = 0; c < NIN; ++c) s[c] = in[c * n + v];
        store8(X + v * C_IN, s);
        const float z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        store8(X + v * C_IN + 8, z);
    }
}

template <int C0>
__device__ __forceinline__ float head_dot(const bf16* a, const float* w, float b, float* av) {
    float o = b;
#pragma unroll
    for (int h = 0; h < C0 / 8; ++h) {
        const bf8 q = load8(a + 8 * h);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            av[8 * h + e] = q.v[e];
            o += q.v[e] * w[8 * h + e];
        }
    }
    return o;
}

// Inference head: delta[v] (FP64) = (sum_c A[v][c] w[c] + b) * scale.
template <int C0>
__global__ void k_head_infer(long long n, const bf16* __restrict__ A, const float* __restrict__ wb, double scale,
                             double* __restrict__ delta, const double* __restrict__ scal = nullptr) {
    if (scal) scale = scal[2];   // the device-computed output scale (k_net_scales)
    __shared__ float w[C0 + 1];
    if (threadIdx.x <= C0) w[threadIdx.x] = wb[threadIdx.x];
    __syncthreads();
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float av[C0];
        delta[v] = (double)head_dot<C0>(A + v * C0, w, w[C0], av) * scale;
    }
}

constexpr int HEAD_THREADS = 256;
template <int C0>
__host__ __device__ constexpr int head_len() {
    return C0 + 2;   // dw[C0], db, sum of squared errors
}

// Training head: loss and its gradient.  out = A.w + b, e = out - t*tscale,
// dOut = 2e/n; G[v][c] = bf16(dOut w[c] leaky'(A)); per-block partials of
// dw (C0), db and sum e^2; out written when `out` is not null.
template <int C0>
__global__ void __launch_bounds__(HEAD_THREADS) k_head_train(long long n, const bf16* __restrict__ A,
                                                             const float* __restrict__ wb, const float* __restrict__ t,
                                                             float tscale, float slope, bf16* __restrict__ G,
                                                             float* __restrict__ part, float* __restrict__ out) {
    __shared__ float w[C0 + 1];
    __shared__ float red[HEAD_THREADS / 32][head_len<C0>()];
    if (threadIdx.x <= C0) w[threadIdx.x] = wb[threadIdx.x];
    __syncthreads();
    float acc[head_len<C0>()];
#pragma unroll
    for (int i = 0; i < head_len<C0>(); ++i) acc[i] = 0.f;
    const float inv_n2 = 2.0f / (float)n;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float av[C0];
        const float o = head_dot<C0>(A + v * C0, w, w[C0], av);
        if (out) out[v] = o;
        const float e = o - t[v] * tscale;
        const float dO = e * inv_n2;
        float gv[C0];
#pragma unroll
        for (int c = 0; c < C0; ++c) {
            acc[c] += av[c] * dO;
            gv[c] = dO * w[c] * (av[c] > 0.f ? 1.f : slope);
        }
#pragma unroll
        for (int h = 0; h < C0 / 8; ++h) store8(G + v * C0 + 8 * h, gv + 8 * h);
        acc[C0] += dO;
        acc[C0 + 1] += e * e;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < head_len<C0>(); ++i) {
        float x = acc[i];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][i] = x;
    }
    __syncthreads();
    if (threadIdx.x < head_len<C0>()) {
        float s = 0.f;
        for (int wi = 0; wi < HEAD_THREADS / 32; ++wi) s += red[wi][threadIdx.x];
        part[(long long)blockIdx.x * head_len<C0>() + threadIdx.x] = s;
    }
}

// Divergence of (u, v, w) per cell, as the residual norms define it, into
// raw (FP32); per-block partials of sum div^2 and sum dp1^2.
__global__ void __launch_bounds__(256) k_div_field(mdx_dims d, int pery, double idx, double idy, double idz,
                                                   const double* __restrict__ u, const double* __restrict__ v,
                                                   const double* __restrict__ w, const double* __restrict__ dp1,
                                                   float* __restrict__ raw, double* __restrict__ part) {
    double s0 = 0.0, s1 = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int j = (int)(r % d.ny) + 1;
        const int k = (int)(r / d.ny) + 1;
        const int ip = i + 1 > d.nx ? 1 : i + 1;
        const int jp = (pery && j + 1 > d.ny) ? 1 : j + 1;
        const int kp = k + 1 > d.nz ? 1 : k + 1;
        const long long c = pidx(d, i, j, k);
        const double dv = (__ldg(u + pidx(d, ip, j, k)) - __ldg(u + c)) * idx +
                          (__ldg(v + pidx(d, i, jp, k)) - __ldg(v + c)) * idy +
                          (__ldg(w + pidx(d, i, j, kp)) - __ldg(w + c)) * idz;
        raw[t] = (float)dv;
        s0 += dv * dv;
        const double q = __ldg(dp1 + t);
        s1 += q * q;
    }
    __shared__ double sh[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = s0;
        sh[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int i = 0; i < 8; ++i) s += sh[threadIdx.x][i];
        part[2 * blockIdx.x + threadIdx.x] = s;
    }
}

// Per-block partial sums of a double field (pairs: sum, 0), grid-stride so
// that the block count, and with it the summation order, is fixed.
__global__ void __launch_bounds__(256) k_sum_field(long long n, const double* __restrict__ a,
                                                   double* __restrict__ part) {
    double s0 = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        s0 += a[t];
    __shared__ double sh[8];
    for (int o = 16; o > 0; o >>= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s0;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < 8; ++i) s += sh[i];
        part[2 * blockIdx.x] = s;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// Along a correction delta applied once: per-block pairs of sum(delta d0)
// and sum(delta (d1 - d0)), d0 = raw (the divergence before, FP32), d1 the
// divergence of (u, v, w) now (the red-black neighbour rule).  With A =
// -div(mu grad), applying delta changes the divergence by dt_gamma A delta =
// d1 - d0, so -sum(delta d0) / sum(delta (d1 - d0)) is the step along delta
// that minimises the energy norm of the pressure error.
__global__ void __launch_bounds__(256) k_energy_dots(mdx_dims d, int pery, double idx, double idy, double idz,
                                                     const double* __restrict__ u, const double* __restrict__ v,
                                                     const double* __restrict__ w, const float* __restrict__ raw,
                                                     const double* __restrict__ delta, double* __restrict__ part) {
    double s0 = 0.0, s1 = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < d.nint; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % d.nx) + 1;
        const long long r = t / d.nx;
        const int j = (int)(r % d.ny) + 1;
        const int k = (int)(r / d.ny) + 1;
        const int ip = i + 1 > d.nx ? 1 : i + 1;
        const int jp = (pery && j + 1 > d.ny) ? 1 : j + 1;
        const int kp = k + 1 > d.nz ? 1 : k + 1;
        const long long c = pidx(d, i, j, k);
        const double d1 = (__ldg(u + pidx(d, ip, j, k)) - __ldg(u + c)) * idx +
                          (__ldg(v + pidx(d, i, jp, k)) - __ldg(v + c)) * idy +
                          (__ldg(w + pidx(d, i, j, kp)) - __ldg(w + c)) * idz;
        const double d0 = (double)raw[t], dl = __ldg(delta + t);
        s0 += dl * d0;
        s1 += dl * (d1 - d0);
    }
    __shared__ double sh[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = s0;
        sh[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double q = 0.0;
        for (int i = 0; i < 8; ++i) q += sh[threadIdx.x][i];
        part[2 * blockIdx.x + threadIdx.x] = q;
    }
}

__global__ void k_scale(long long n, double* __restrict__ a, double c) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a[t] *= c;
}

__global__ void k_add_const(long long n, double* __restrict__ a, double c) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a[t] += c;
}

// Sum of n-block pairs -> out[0..1] (one block).
__global__ void k_sum_pairs(int nb, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[2][256];
    double s0 = 0.0, s1 = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        s0 += part[2 * b];
        s1 += part[2 * b + 1];
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = s1;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + h];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sh[0][0];
        out[1] = sh[1][0];
    }
}

// Normalised inputs: in[0] = raw*ir, in[1] = dp1*ip, in[2] = dp2*ip, in[3] =
// IBM factor of the cell (mean of its three lower faces; 1 without IBM),
// in[4] = vis, the same for every cell (net_vis_input: the flow's viscous
// number).  DEV: the two scales come from the device (scal[0], scal[1]),
// written by k_net_scales, so that the pass needs no host read.
template <bool DEV>
__global__ void k_norm_in_t(mdx_dims d, int mu_mode, const float* __restrict__ raw, const double* __restrict__ dp1,
                            const double* __restrict__ dp2, const double* __restrict__ mu, double ir, double ip,
                            float vis, const double* __restrict__ scal, float* __restrict__ in) {
    if (DEV) {
        ir = scal[0];
        ip = scal[1];
    }
    const long long n = d.nint;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        in[t] = (float)(raw[t] * ir);
        in[n + t] = (float)(dp1[t] * ip);
        in[2 * n + t] = (float)(dp2[t] * ip);
        float m = 1.f;
        if (mu_mode != 0) {
            const int i = (int)(t % d.nx) + 1;
            const long long r = t / d.nx;
            const int j = (int)(r % d.ny) + 1;
            const int k = (int)(r / d.ny) + 1;
            double a, b, c;
            if (mu_mode == 1) {
                const long long np = (long long)d.nxp * d.nyp, q = i + (long long)d.nxp * j;
                a = mu[q];
                b = mu[np + q];
                c = mu[2 * np + q];
            } else {
                const long long q = pidx(d, i, j, k);
                a = mu[q];
                b = mu[d.npad + q];
                c = mu[2 * d.npad + q];
            }
            m = (float)((a + b + c) * (1.0 / 3.0));
        }
        in[3 * n + t] = m;
        in[4 * n + t] = vis;
    }
}

// The network's constant input: the viscous number dt_gamma / (Re h^2) of
// the substage, as log10 + 3 (about -0.8 .. 0.6 over Re 1000..5000 on the
// 256x128x128 channel at dt 1e-3).  The pressure increment's shape depends
// on how far viscous diffusion reaches in a substage; the other inputs are
// normalised and carry no scale.
float net_vis_input(double dg, double ire, double h2) {
    const double v = std::fabs(dg) * ire / h2;
    return v > 0.0 && std::isfinite(v) ? (float)(std::log10(v) + 3.0) : 0.f;
}

// Input and output scales of one pass from the sums of div^2 and dp1^2 over
// n cells (sums[0..1]): scal = {1/rms(div), 1/rms(dp1) (1 when 0), the
// output scale out_scale rms(div) h^2 / dt_gamma}; *ok = 0 when the
// divergence is zero or not finite (no correction).
__global__ void k_net_scales(long long n, const double* __restrict__ sums, double out_scale, double h2, double dg,
                             double* __restrict__ scal, int* __restrict__ ok) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double sr = sqrt(sums[0] / (double)n);
    double sp = sqrt(sums[1] / (double)n);
    const bool good = sr > 0.0 && isfinite(sr);
    if (!(sp > 0.0) || !isfinite(sp)) sp = 1.0;
    scal[0] = good ? 1.0 / sr : 0.0;
    scal[1] = 1.0 / sp;
    scal[2] = good ? out_scale * sr * h2 / dg : 0.0;
    *ok = good ? 1 : 0;
}

// a[t] -= sums[0] / n (the mean from k_sum_pairs)
__global__ void k_sub_mean(long long n, double* __restrict__ a, const double* __restrict__ sums) {
    const double m = sums[0] / (double)n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a[t] -= m;
}

// Snapshot target: (dp - g) * scale.
__global__ void k_snap_target(long long n, const double* __restrict__ dp, const double* __restrict__ g, double scale,
                              float* __restrict__ t) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        t[v] = (float)((dp[v] - g[v]) * scale);
}

// Per-block partial of sum t^2 (pairs, second slot 0).
__global__ void __launch_bounds__(256) k_sumsq(long long n, const float* __restrict__ t, double* __restrict__ part) {
    double s = 0.0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const double q = t[v];
        s += q * q;
    }
    __shared__ double sh[8];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int i = 0; i < 8; ++i) a += sh[i];
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// Adam on the flat FP32 parameters.
__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// BF16 copies of one convolution's weights: Wf[tap][co][ci] and
// Wt[26-tap][ci][co].
__global__ void k_export_w(int cin, int cout, const float* __restrict__ w, bf16* __restrict__ wf, bf16* __restrict__ wt) {
    const int n = 27 * cout * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int tap = i / (cout * cin), r = i - tap * cout * cin;
        const int co = r / cin, ci = r - co * cin;
        const bf16 b = __float2bfloat16_rn(w[i]);
        wf[i] = b;
        wt[((26 - tap) * cin + ci) * cout + co] = b;
    }
}

// ---- host side -------------------------------------------------------------

struct conv_layer {
    int cin, cout, level;
    long long w_off, b_off;   // into the flat parameter vector
    bf16* wf = nullptr;
    bf16* wt = nullptr;
};

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t& s) {
    return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

struct mdx_unet {
    mdx_unet_opts_t o{};
    lvl L[4]{};
    int c0 = 16, c1 = 32, pery = 0;
    std::vector<conv_layer> conv;   // enc0a enc0b enc1a enc1b enc2a enc2b enc3a enc3b extra... dec2 dec1 dec0
    long long head_off = 0, nparam = 0;
    float *param = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    int adam_t = 0;
    // activations (BF16): x0, per-conv outputs, pools, up-adds
    bf16* x0 = nullptr;
    std::vector<bf16*> act;   // one per conv layer
    bf16* pool[4] = {nullptr, nullptr, nullptr, nullptr};   // pool[l]: input of level l (l >= 1)
    bf16* up[3] = {nullptr, nullptr, nullptr};              // up[l]: up(..) + skip at level l
    // gradients
    float* dU[3] = {nullptr, nullptr, nullptr};             // FP32, gradient of up[l]
    float* dP[4] = {nullptr, nullptr, nullptr, nullptr};    // FP32, gradient of pool[l]
    float* dT[4] = {nullptr, nullptr, nullptr, nullptr};    // FP32, gradient of a conv input at level l
    bf16* G[4] = {nullptr, nullptr, nullptr, nullptr};      // BF16, pre-activation gradient at level l
    float* part = nullptr;                                  // weight-gradient partials
    int part_blocks = 0;
    float* head_part = nullptr;
    int head_blocks = 0;
    float* out = nullptr;       // FP32 head output (training)
    float* in = nullptr;        // [NIN][n] normalised inputs (inference)
    float* raw = nullptr;       // raw divergence
    double* delta = nullptr;    // learned correction
    double* red_part = nullptr;
    double* red_out = nullptr;
    double* red_host = nullptr;
    int red_blocks = 0;
    // snapshots: slot s holds in[NIN][n] then target[n]
    float* snap = nullptr;
    int stored = 0, next = 0;
    long long total_snaps = 0;
    int pending = -1;           // slot awaiting its target
    double pending_scale = 0.0;
    bool recording = false, trained = false;
    double out_scale = 1.0;
    uint64_t order_state = 0;
    mdx_unet_stats_t st{};
    // gate (o.gate_period > 0): per RK substage, exponential averages of the
    // iterations of projections with the correction (on) and with the
    // extrapolated guess alone (off), their sample counts, projections since
    // the other arm was last tried, and this projection's arm (-1: none)
    double gate_ema[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    int gate_n[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    int gate_since[3] = {0, 0, 0};
    int gate_arm = -1;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int* tc_err = nullptr;      // set by a tcgen05 convolution whose bounded wait gave up
};

namespace {

// tcgen05 convolution: output rows per CTA (4 for 16 input channels, 2 for
// 32: four staged planes then fill most of shared memory) and z planes per
// CTA (4 for the 16->16 layers, 8 where the staged weights are larger),
// measured on the C1 level sizes.
template <int CIN, int COUT>
struct tc_cfg {
    static constexpr int RY = CIN == 16 ? 4 : 2;
    static constexpr int ZC = CIN * COUT >= 512 ? 8 : 4;
};

template <int CIN, int COUT>
int set_attrs(mdx_ctx_t* ctx) {
    using R = tc_cfg<CIN, COUT>;
    constexpr int tsmem = tc::pgeom<CIN, COUT, R::RY>::SMEM;
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_conv3_tcp<CIN, COUT, 0, R::RY, lvl>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_conv3_tcp<CIN, COUT, 1, R::RY, lvl>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, tsmem));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_conv3<CIN, COUT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       conv_smem<CIN, COUT>()));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_conv3<CIN, COUT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       conv_smem<CIN, COUT>()));
    MDX_CUDA(ctx, cudaFuncSetAttribute(k_conv3_wgrad<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       wgrad_smem<CIN, COUT>()));
    return MDX_OK;
}

int nblocks(long long work, int threads = 256, int cap = 8192) {
    return (int)std::max<long long>(1, std::min<long long>((work + threads - 1) / threads, cap));
}

int ntiles_host(const lvl& L) {
    return ((L.nx + TX - 1) / TX) * ((L.ny + TY - 1) / TY) * ((L.nz + TZ - 1) / TZ);
}

template <int CIN, int COUT, int EPI>
int conv_launch(mdx_ctx_t* ctx, mdx_unet* U, const lvl& L, int pery, const bf16* X, const bf16* W, const float* b,
                float slope, bf16* Yb, float* Yf) {
    if (U->o.conv_kernel == 0 && L.nx % tc::XT == 0) {   // tcgen05, whole 128-voxel rows
        using R = tc_cfg<CIN, COUT>;
        auto tfn = k_conv3_tcp<CIN, COUT, EPI, R::RY, lvl>;
        constexpr int tsmem = tc::pgeom<CIN, COUT, R::RY>::SMEM;
        const dim3 grid(L.nx / tc::XT, (L.ny + R::RY - 1) / R::RY, (L.nz + R::ZC - 1) / R::ZC);
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet conv tc", tfn, grid, tc::THREADS, tsmem, L, pery, R::ZC, X, W, b, slope,
                   Yb, Yf, U->tc_err);
        U->st.tc_convs++;
        return MDX_OK;
    }
    auto kfn = k_conv3<CIN, COUT, EPI>;
    constexpr int smem = conv_smem<CIN, COUT>();
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet conv", kfn, ntiles_host(L), 256, smem, L, pery, X, W, b, slope, Yb, Yf);
    return MDX_OK;
}

// Forward (EPI 0) or data gradient (EPI 1, transposed weights) of a conv.
int conv_run(mdx_ctx_t* ctx, mdx_unet* U, const conv_layer& c, bool data_grad, const bf16* X, bf16* Yb, float* Yf) {
    const lvl& L = U->L[c.level];
    const float slope = (float)U->o.slope;
    const float* b = U->param + c.b_off;
    const int ci = data_grad ? c.cout : c.cin, co = data_grad ? c.cin : c.cout;
    const bf16* W = data_grad ? c.wt : c.wf;
#define MDX_CONV_CASE(A, B)                                                                               \
    if (ci == A && co == B)                                                                               \
        return data_grad ? conv_launch<A, B, 1>(ctx, U, L, U->pery, X, W, b, slope, Yb, Yf)               \
                         : conv_launch<A, B, 0>(ctx, U, L, U->pery, X, W, b, slope, Yb, Yf);
    MDX_CONV_CASE(16, 16)
    MDX_CONV_CASE(16, 32)
    MDX_CONV_CASE(32, 16)
    MDX_CONV_CASE(32, 32)
#undef MDX_CONV_CASE
    return mdx_fail(ctx, MDX_ERR_ARG, "unet: unsupported channel pair %d -> %d", ci, co);
}

template <int CIN, int COUT>
int wgrad_launch(mdx_ctx_t* ctx, mdx_unet* U, const conv_layer& c, const bf16* X, const bf16* Gd) {
    const lvl& L = U->L[c.level];
    const int nb = std::min(ntiles_host(L), U->part_blocks);
    constexpr int len = wgrad_len<CIN, COUT>();
    auto kfn = k_conv3_wgrad<CIN, COUT>;
    constexpr int nth = wgrad_warps<CIN, COUT>() * 32, smem = wgrad_smem<CIN, COUT>();
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet wgrad", kfn, nb, nth, smem, L, U->pery, X, Gd, U->part);
    // W block then bias block: both contiguous in the parameter layout
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet wgrad sum", k_sum_parts, (len + 255) / 256, 256, 0, nb, len, U->part,
               U->grad + c.w_off);
    return MDX_OK;
}

int wgrad_run(mdx_ctx_t* ctx, mdx_unet* U, const conv_layer& c, const bf16* X, const bf16* Gd) {
    if (c.cin == 16 && c.cout == 16) return wgrad_launch<16, 16>(ctx, U, c, X, Gd);
    if (c.cin == 16 && c.cout == 32) return wgrad_launch<16, 32>(ctx, U, c, X, Gd);
    if (c.cin == 32 && c.cout == 16) return wgrad_launch<32, 16>(ctx, U, c, X, Gd);
    if (c.cin == 32 && c.cout == 32) return wgrad_launch<32, 32>(ctx, U, c, X, Gd);
    return mdx_fail(ctx, MDX_ERR_ARG, "unet: unsupported channel pair");
}

int n_enc(const mdx_unet* U) {
    return 8 + U->o.extra_bottleneck;   // convs before the decoder
}

// Forward pass from U->x0; the output activation of dec0 is act.back().
int forward(mdx_ctx_t* ctx, mdx_unet* U) {
    const int ne = n_enc(U);
    auto& c = U->conv;
    auto& A = U->act;
    const int C[4] = {U->c0, U->c1, U->c1, U->c1};
    MDX_TRY(conv_run(ctx, U, c[0], false, U->x0, A[0], nullptr));
    MDX_TRY(conv_run(ctx, U, c[1], false, A[0], A[1], nullptr));
    for (int l = 1; l <= 3; ++l) {
        const bf16* skip = A[2 * l - 1];
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet pool", k_pool, nblocks(U->L[l].n * C[l - 1] / 8), 256, 0, U->L[l],
                   U->L[l - 1], C[l - 1], skip, U->pool[l]);
        MDX_TRY(conv_run(ctx, U, c[2 * l], false, U->pool[l], A[2 * l], nullptr));
        MDX_TRY(conv_run(ctx, U, c[2 * l + 1], false, A[2 * l], A[2 * l + 1], nullptr));
    }
    for (int e = 8; e < ne; ++e) MDX_TRY(conv_run(ctx, U, c[e], false, A[e - 1], A[e], nullptr));
    // decoder: dec2 (ne), dec1 (ne+1), dec0 (ne+2)
    const bf16* below = A[ne - 1];
    for (int l = 2; l >= 0; --l) {
        const int li = ne + (2 - l);
        const bf16* skip = A[2 * l + 1];
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet up", k_up_add, nblocks(U->L[l].n * C[l] / 8), 256, 0, U->L[l], U->L[l + 1],
                   C[l], below, skip, U->up[l]);
        MDX_TRY(conv_run(ctx, U, c[li], false, U->up[l], A[li], nullptr));
        below = A[li];
    }
    return MDX_OK;
}

// Backward pass from G[0] = gradient at the pre-activation of dec0.
int backward(mdx_ctx_t* ctx, mdx_unet* U) {
    const int ne = n_enc(U);
    auto& c = U->conv;
    auto& A = U->act;
    const int C[4] = {U->c0, U->c1, U->c1, U->c1};
    const float slope = (float)U->o.slope;
    // decoder, finest first: dec0 at level 0 .. dec2 at level 2
    for (int l = 0; l <= 2; ++l) {
        const int li = ne + (2 - l);
        MDX_TRY(wgrad_run(ctx, U, c[li], U->up[l], U->G[l]));
        MDX_TRY(conv_run(ctx, U, c[li], true, U->G[l], nullptr, U->dU[l]));
        // gradient of the layer below the up-add (the next decoder conv or the bottleneck output)
        const int below = (l < 2) ? ne + (2 - (l + 1)) : ne - 1;
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet act bwd down", k_act_bwd_down, nblocks(U->L[l + 1].n * C[l] / 8), 256, 0,
                   U->L[l + 1], U->L[l], C[l], U->dU[l], A[below], slope, U->G[l + 1]);
    }
    // bottleneck at level 3: layers ne-1 .. 6
    for (int li = ne - 1; li >= 6; --li) {
        const bf16* X = (li == 6) ? U->pool[3] : A[li - 1];
        MDX_TRY(wgrad_run(ctx, U, c[li], X, U->G[3]));
        if (li == 6) {
            MDX_TRY(conv_run(ctx, U, c[li], true, U->G[3], nullptr, U->dP[3]));
        } else {
            MDX_TRY(conv_run(ctx, U, c[li], true, U->G[3], nullptr, U->dT[3]));
            MDX_LAUNCH(ctx, MDX_T_OTHER, "unet act bwd", k_act_bwd_same, nblocks(U->L[3].n * C[3] / 8), 256, 0, U->L[3],
                       U->L[3], C[3], U->dT[3], (const float*)nullptr, A[li - 1], slope, U->G[3]);
        }
    }
    // encoder levels 2, 1, 0: b-conv output gets dU[l] (skip) + dP[l+1]/8 (pool)
    for (int l = 2; l >= 0; --l) {
        const int lb = 2 * l + 1, la = 2 * l;
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet act bwd", k_act_bwd_same, nblocks(U->L[l].n * C[l] / 8), 256, 0, U->L[l],
                   U->L[l + 1], C[l], U->dU[l], U->dP[l + 1], A[lb], slope, U->G[l]);
        MDX_TRY(wgrad_run(ctx, U, c[lb], A[la], U->G[l]));
        MDX_TRY(conv_run(ctx, U, c[lb], true, U->G[l], nullptr, U->dT[l]));
        const int cin_a = c[la].cout;
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet act bwd", k_act_bwd_same, nblocks(U->L[l].n * cin_a / 8), 256, 0, U->L[l],
                   U->L[l], cin_a, U->dT[l], (const float*)nullptr, A[la], slope, U->G[l]);
        const bf16* Xa = (l == 0) ? U->x0 : U->pool[l];
        MDX_TRY(wgrad_run(ctx, U, c[la], Xa, U->G[l]));
        if (l > 0) MDX_TRY(conv_run(ctx, U, c[la], true, U->G[l], nullptr, U->dP[l]));
    }
    return MDX_OK;
}

int export_weights(mdx_ctx_t* ctx, mdx_unet* U) {
    for (auto& c : U->conv)
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet export", k_export_w, nblocks(27LL * c.cin * c.cout), 256, 0, c.cin, c.cout,
                   U->param + c.w_off, c.wf, c.wt);
    return MDX_OK;
}

int head_train(mdx_ctx_t* ctx, mdx_unet* U, const float* target, float tscale, float* out) {
    const long long n = U->L[0].n;
    const int nb = U->head_blocks;
    constexpr int len = head_len<16>();
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet head", k_head_train<16>, nb, HEAD_THREADS, 0, n, U->act.back(),
               U->param + U->head_off, target, tscale, (float)U->o.slope, U->G[0], U->head_part, out);
    // dw (16) and db land at head_off; the squared error after them
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet head sum", k_sum_parts, 1, 32, 0, nb, len, U->head_part, U->out);
    MDX_CUDA(ctx, cudaMemcpyAsync(U->grad + U->head_off, U->out, sizeof(float) * (len - 1), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
    return MDX_OK;
}

int pairs_to_host(mdx_ctx_t* ctx, mdx_unet* U, int nb, double* a, double* b) {
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet sum pairs", k_sum_pairs, 1, 256, 0, nb, U->red_part, U->red_out);
    MDX_CUDA(ctx, cudaMemcpyAsync(U->red_host, U->red_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *a = U->red_host[0];
    if (b) *b = U->red_host[1];
    return MDX_OK;
}

template <typename T>
int dalloc(mdx_ctx_t* ctx, T** p, long long n) {
    MDX_CUDA(ctx, cudaMalloc(p, sizeof(T) * (size_t)std::max<long long>(n, 1)));
    return MDX_OK;
}

double h2_of(const mdx_ctx_t* ctx) {
    const mdx_grid_t& g = ctx->g;
    return 1.0 / (1.0 / (g.dx * g.dx) + 1.0 / (g.dy * g.dy) + 1.0 / (g.dz * g.dz));
}

int need_unet(mdx_ctx_t* ctx) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!ctx->unet) return mdx_fail(ctx, MDX_ERR_STATE, "no network: call mdx_unet_create first");
    return MDX_OK;
}

int alloc_net(mdx_ctx_t* ctx, mdx_unet* U) {
    const long long n0 = U->L[0].n;
    MDX_TRY(dalloc(ctx, &U->param, U->nparam));
    MDX_TRY(dalloc(ctx, &U->grad, U->nparam));
    MDX_TRY(dalloc(ctx, &U->adam_m, U->nparam));
    MDX_TRY(dalloc(ctx, &U->adam_v, U->nparam));
    MDX_CUDA(ctx, cudaMemsetAsync(U->grad, 0, sizeof(float) * U->nparam, ctx->stream));
    MDX_CUDA(ctx, cudaMemsetAsync(U->adam_m, 0, sizeof(float) * U->nparam, ctx->stream));
    MDX_CUDA(ctx, cudaMemsetAsync(U->adam_v, 0, sizeof(float) * U->nparam, ctx->stream));
    for (auto& c : U->conv) {
        MDX_TRY(dalloc(ctx, &c.wf, 27LL * c.cin * c.cout));
        MDX_TRY(dalloc(ctx, &c.wt, 27LL * c.cin * c.cout));
    }
    MDX_TRY(dalloc(ctx, &U->x0, n0 * C_IN));
    U->act.assign(U->conv.size(), nullptr);
    for (size_t i = 0; i < U->conv.size(); ++i)
        MDX_TRY(dalloc(ctx, &U->act[i], U->L[U->conv[i].level].n * U->conv[i].cout));
    const int C[4] = {U->c0, U->c1, U->c1, U->c1};
    for (int l = 1; l <= 3; ++l) MDX_TRY(dalloc(ctx, &U->pool[l], U->L[l].n * C[l - 1]));
    for (int l = 0; l <= 2; ++l) {
        MDX_TRY(dalloc(ctx, &U->up[l], U->L[l].n * C[l]));
        MDX_TRY(dalloc(ctx, &U->dU[l], U->L[l].n * C[l]));
    }
    for (int l = 1; l <= 3; ++l) MDX_TRY(dalloc(ctx, &U->dP[l], U->L[l].n * C[l - 1]));
    for (int l = 0; l <= 3; ++l) {
        const int cmax = std::max(C[l], l > 0 ? C[l - 1] : C[l]);
        MDX_TRY(dalloc(ctx, &U->dT[l], U->L[l].n * cmax));
        MDX_TRY(dalloc(ctx, &U->G[l], U->L[l].n * cmax));
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
    U->part_blocks = std::max(dev_sms, 1);
    MDX_TRY(dalloc(ctx, &U->part, (long long)U->part_blocks * (27 * 32 * 32 + 32)));
    U->head_blocks = std::min<long long>(1024, (n0 + HEAD_THREADS - 1) / HEAD_THREADS);
    MDX_TRY(dalloc(ctx, &U->head_part, (long long)U->head_blocks * head_len<16>()));
    MDX_TRY(dalloc(ctx, &U->out, std::max<long long>(n0, 64)));
    MDX_TRY(dalloc(ctx, &U->in, NIN * n0));
    MDX_TRY(dalloc(ctx, &U->raw, n0));
    MDX_TRY(dalloc(ctx, &U->delta, n0));
    U->red_blocks = std::min<long long>(1024, (n0 + 255) / 256);
    MDX_TRY(dalloc(ctx, &U->red_part, 2LL * U->red_blocks));
    MDX_TRY(dalloc(ctx, &U->red_out, 2));
    MDX_CUDA(ctx, cudaMallocHost(&U->red_host, 2 * sizeof(double)));
    if (U->o.capacity > 0) MDX_TRY(dalloc(ctx, &U->snap, (long long)U->o.capacity * (NIN + 1) * n0));
    MDX_CUDA(ctx, cudaEventCreate(&U->ev[0]));
    MDX_CUDA(ctx, cudaEventCreate(&U->ev[1]));
    MDX_CUDA(ctx, cudaMalloc(&U->tc_err, sizeof(int)));
    MDX_CUDA(ctx, cudaMemsetAsync(U->tc_err, 0, sizeof(int), ctx->stream));
    MDX_TRY((set_attrs<16, 16>(ctx)));
    MDX_TRY((set_attrs<16, 32>(ctx)));
    MDX_TRY((set_attrs<32, 16>(ctx)));
    MDX_TRY((set_attrs<32, 32>(ctx)));
    return MDX_OK;
}

// One forward + head + backward on the inputs in4 (device, [4][n]) and
// target t (device) scaled by tscale; leaves the gradient in U->grad and the
// mean squared error in U->out[head_len-1] / n.
int loss_grad(mdx_ctx_t* ctx, mdx_unet* U, const float* in4, const float* t, float tscale, float* out) {
    const long long n0 = U->L[0].n;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet pack", k_pack_in, nblocks(n0), 256, 0, n0, in4, U->x0);
    MDX_TRY(forward(ctx, U));
    MDX_TRY(head_train(ctx, U, t, tscale, out));
    MDX_TRY(backward(ctx, U));
    return MDX_OK;
}

// A tcgen05 convolution whose bounded wait gave up leaves *tc_err set: read
// it (synchronising) where the caller synchronises anyway.
int check_tc(mdx_ctx_t* ctx, mdx_unet* U) {
    int e = 0;
    MDX_CUDA(ctx, cudaMemcpyAsync(&e, U->tc_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (e) return mdx_fail(ctx, MDX_ERR_TIMEOUT, "unet: a tensor-core convolution timed out waiting for its MMAs");
    return MDX_OK;
}

}  // namespace

void mdx_unet_free(mdx_ctx_t* ctx) {
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (!U) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto& c : U->conv) {
        cudaFree(c.wf);
        cudaFree(c.wt);
    }
    for (auto* p : U->act) cudaFree(p);
    for (int l = 0; l < 4; ++l) {
        cudaFree(U->pool[l]);
        cudaFree(U->dP[l]);
        cudaFree(U->dT[l]);
        cudaFree(U->G[l]);
    }
    for (int l = 0; l < 3; ++l) {
        cudaFree(U->up[l]);
        cudaFree(U->dU[l]);
    }
    cudaFree(U->x0);
    cudaFree(U->param);
    cudaFree(U->grad);
    cudaFree(U->adam_m);
    cudaFree(U->adam_v);
    cudaFree(U->part);
    cudaFree(U->head_part);
    cudaFree(U->out);
    cudaFree(U->in);
    cudaFree(U->raw);
    cudaFree(U->delta);
    cudaFree(U->red_part);
    cudaFree(U->red_out);
    cudaFreeHost(U->red_host);
    cudaFree(U->snap);
    if (U->ev[0]) cudaEventDestroy(U->ev[0]);
    if (U->ev[1]) cudaEventDestroy(U->ev[1]);
    cudaFree(U->tc_err);
    delete U;
    ctx->unet = nullptr;
}

// With the extrapolated increment applied (*rg = ||div u||): record a
// snapshot's inputs, and in learned mode apply the network's correction,
// undoing it when it does not lower ||div u||.  With a gate period the
// correction is applied or not per RK substage by the iterations each
// choice took (mdx_unet_finish records them).
int mdx_unet_correct(mdx_ctx_t* ctx, double dg, double* rg) {
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    const bool learn = ctx->guess_mode == MDX_GUESS_LEARNED && U->trained;
    const bool rec = U->recording && U->o.capacity > 0 && ctx->opts.tol > 0.0;
    if (!learn && !rec) return MDX_OK;
    const mdx_dims& d = ctx->d;
    const long long n = d.nint;
    const int s = (int)(ctx->proj_count % 3);
    // the gate: off -> the extrapolated guess alone for this projection
    bool apply = learn;
    U->gate_arm = -1;
    if (learn && U->o.gate_period > 0) {
        const int* cnt = U->gate_n[s];
        int arm;
        if (cnt[0] == 0) arm = 0;        // a baseline without the correction first
        else if (cnt[1] == 0) arm = 1;
        else {
            const int pref = U->gate_ema[s][1] <= U->gate_ema[s][0] ? 1 : 0;
            arm = pref;
            if (++U->gate_since[s] >= U->o.gate_period) {   // re-try the other arm
                arm = 1 - pref;
                U->gate_since[s] = 0;
            }
        }
        U->gate_arm = arm;
        if (arm == 0) {
            apply = false;
            U->st.gated++;
        }
    }
    if (!apply && !rec) return MDX_OK;
    if (apply) MDX_CUDA(ctx, cudaEventRecord(U->ev[0], ctx->stream));
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet div field", k_div_field, U->red_blocks, 256, 0, d, U->pery, 1.0 / ctx->g.dx,
               1.0 / ctx->g.dy, 1.0 / ctx->g.dz, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN], ctx->dp_hist[s], U->raw,
               U->red_part);
    double sr = 0.0, sp = 0.0;
    MDX_TRY(pairs_to_host(ctx, U, U->red_blocks, &sr, &sp));
    sr = std::sqrt(sr / (double)n);
    sp = std::sqrt(sp / (double)n);
    if (!(sr > 0.0) || !std::isfinite(sr)) return MDX_OK;
    if (!(sp > 0.0) || !std::isfinite(sp)) sp = 1.0;
    const double h2 = h2_of(ctx);
    float* dst = U->in;
    if (rec) {
        dst = U->snap + (long long)U->next * (NIN + 1) * n;
        U->pending = U->next;
        U->pending_scale = dg / (sr * h2);
    }
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet inputs", k_norm_in_t<false>, nblocks(n), 256, 0, d, ctx->mu_mode, U->raw,
               ctx->dp_hist[s], ctx->dp_hist2[s], ctx->mu, 1.0 / sr, 1.0 / sp, net_vis_input(dg, 1.0 / ctx->g.re, h2),
               (const double*)nullptr, dst);
    if (!apply) return MDX_OK;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet pack", k_pack_in, nblocks(n), 256, 0, n, dst, U->x0);
    MDX_TRY(forward(ctx, U));
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet head", k_head_infer<16>, nblocks(n), 256, 0, n, U->act.back(),
               U->param + U->head_off, U->out_scale * sr * h2 / dg, U->delta, (const double*)nullptr);
    // A constant pressure increment moves no face (the red-black operator's
    // null space with periodic or Neumann pressure), so the solve never
    // removes one; a correction with a non-zero mean would shift p by a
    // constant every projection and p would drift from the plain method's
    // by a growing constant.  The correction is therefore made zero-mean.
    {
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet delta mean", k_sum_field, U->red_blocks, 256, 0, n, U->delta, U->red_part);
        double sum = 0.0;
        MDX_TRY(pairs_to_host(ctx, U, U->red_blocks, &sum, nullptr));
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet delta zero mean", k_add_const, nblocks(n), 256, 0, n, U->delta,
                   -sum / (double)n);
    }
    MDX_TRY(mdx_apply_guess(ctx, U->delta, dg));
    bool keep_by_energy = false;
    if (U->o.step_rule == 1) {
        // the energy-optimal step alpha along delta: apply (alpha - 1) delta
        // more; kept when alpha > 0 (the error's energy norm then falls)
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet energy dots", k_energy_dots, U->red_blocks, 256, 0, d, U->pery,
                   1.0 / ctx->g.dx, 1.0 / ctx->g.dy, 1.0 / ctx->g.dz, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN],
                   U->raw, U->delta, U->red_part);
        double a = 0.0, b = 0.0;
        MDX_TRY(pairs_to_host(ctx, U, U->red_blocks, &a, &b));
        const double alpha = (b != 0.0) ? -a / b : 0.0;
        U->st.last_step = alpha;
        if (std::isfinite(alpha) && alpha > 0.0) {
            keep_by_energy = true;
            if (alpha != 1.0) {
                MDX_LAUNCH(ctx, MDX_T_OTHER, "unet step scale", k_scale, nblocks(n), 256, 0, n, U->delta, alpha - 1.0);
                MDX_TRY(mdx_apply_guess(ctx, U->delta, dg));
            }
        }
    }
    MDX_CUDA(ctx, cudaEventRecord(U->ev[1], ctx->stream));
    double r = 0.0, linf = 0.0;
    MDX_TRY(mdx_k_div_norms(ctx, ctx->f[MDX_UN], ctx->f[MDX_VN], ctx->f[MDX_WN], &r, &linf));
    MDX_TRY(check_tc(ctx, U));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, U->ev[0], U->ev[1]) == cudaSuccess) U->st.infer_ms = ms;
    if (U->o.step_rule == 1 ? keep_by_energy : r < *rg) {
        U->st.corrections++;
        U->st.last_gain = r > 0.0 ? *rg / r : 0.0;
        *rg = r;
    } else {   // back to the extrapolated guess alone
        U->st.rejected++;
        U->st.last_gain = r > 0.0 ? *rg / r : 0.0;
        MDX_TRY(mdx_undo_guess(ctx));
        MDX_TRY(mdx_apply_guess(ctx, ctx->guess, dg));
    }
    return MDX_OK;
}

// The learned correction for a grid other than the context's -- an ensemble
// member -- with no host read, so that a CUDA graph can hold it: the
// network (sized for the largest member) runs on the member's level sizes
// (the activations are dense [z][y][x][c], so a grid with no more cells at
// every level fits), the scales come from device reductions, and *ok
// (device) says whether delta holds a correction.  Inputs are the member's
// u, v, w after its extrapolated guess, its last two increments of this
// substage and its IBM factor planes (or null).
int mdx_unet_member_delta(mdx_ctx_t* nc, const mdx_dims& dm, double dx, double dy, double dz, double ire, double dg,
                          const double* un, const double* vn, const double* wn, const double* dp1, const double* dp2,
                          const double* mu_planes, double* delta, double* scal, int* ok) {
    mdx_unet* U = static_cast<mdx_unet*>(nc->unet);
    if (!U || !U->trained) return mdx_fail(nc, MDX_ERR_STATE, "ensemble network: no trained parameters");
    if (dm.nx % 8 || dm.ny % 8 || dm.nz % 8) return mdx_fail(nc, MDX_ERR_ARG, "ensemble network: member sizes not multiples of 8");
    if (dm.nint > U->L[0].n) return mdx_fail(nc, MDX_ERR_ARG, "ensemble network: member larger than the network's grid");
    lvl saved[4];
    for (int l = 0; l < 4; ++l) {
        saved[l] = U->L[l];
        U->L[l] = lvl{dm.nx >> l, dm.ny >> l, dm.nz >> l, (long long)(dm.nx >> l) * (dm.ny >> l) * (dm.nz >> l)};
    }
    const long long n = dm.nint;
    const double h2 = 1.0 / (1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz));
    auto run = [&]() -> int {
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet div field", k_div_field, U->red_blocks, 256, 0, dm, U->pery, 1.0 / dx, 1.0 / dy,
                   1.0 / dz, un, vn, wn, dp1, U->raw, U->red_part);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet sum pairs", k_sum_pairs, 1, 256, 0, U->red_blocks, U->red_part, U->red_out);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet scales", k_net_scales, 1, 32, 0, n, U->red_out, U->out_scale, h2, dg, scal, ok);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet inputs", k_norm_in_t<true>, nblocks(n), 256, 0, dm, mu_planes ? 1 : 0, U->raw,
                   dp1, dp2, mu_planes, 0.0, 0.0, net_vis_input(dg, ire, h2), (const double*)scal, U->in);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet pack", k_pack_in, nblocks(n), 256, 0, n, U->in, U->x0);
        MDX_TRY(forward(nc, U));
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet head", k_head_infer<16>, nblocks(n), 256, 0, n, U->act.back(),
                   U->param + U->head_off, 0.0, delta, (const double*)scal);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet delta mean", k_sum_field, U->red_blocks, 256, 0, n, delta, U->red_part);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet sum pairs", k_sum_pairs, 1, 256, 0, U->red_blocks, U->red_part, U->red_out);
        MDX_LAUNCH(nc, MDX_T_OTHER, "unet delta zero mean", k_sub_mean, nblocks(n), 256, 0, n, delta, U->red_out);
        return MDX_OK;
    };
    const int rc = run();
    for (int l = 0; l < 4; ++l) U->L[l] = saved[l];
    return rc;
}

// After the projection (dp_hist[s] = its increment): the pending snapshot's
// target, or drop it when the projection did not converge.
int mdx_unet_finish(mdx_ctx_t* ctx, bool converged, int iterations) {
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (U->gate_arm >= 0) {   // the gate's sample: this projection's iterations
        const int s = (int)(ctx->proj_count % 3), a = U->gate_arm;
        if (converged) {
            double& e = U->gate_ema[s][a];
            e = U->gate_n[s][a] > 0 ? 0.5 * e + 0.5 * (double)iterations : (double)iterations;
            U->gate_n[s][a]++;
        }
        U->gate_arm = -1;
    }
    if (U->pending < 0) return MDX_OK;
    const int slot = U->pending;
    U->pending = -1;
    if (!converged) return MDX_OK;
    const long long n = ctx->d.nint;
    const int s = (int)(ctx->proj_count % 3);
    float* t = U->snap + (long long)slot * (NIN + 1) * n + NIN * n;
    MDX_LAUNCH(ctx, MDX_T_OTHER, "unet snapshot target", k_snap_target, nblocks(n), 256, 0, n, ctx->dp_hist[s],
               ctx->guess, U->pending_scale, t);
    U->next = (U->next + 1) % U->o.capacity;
    U->stored = std::min(U->stored + 1, U->o.capacity);
    U->total_snaps++;
    return MDX_OK;
}

extern "C" {

void mdx_default_unet_opts(mdx_unet_opts_t* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->channels0 = 16;
    o->channels = 32;
    o->extra_bottleneck = 0;
    o->capacity = 64;
    o->slope = 0.1;
    o->seed = 20261203ull;
}

int mdx_unet_create(mdx_ctx_t* ctx, const mdx_unet_opts_t* opts) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    if (!ctx->fields) return mdx_fail(ctx, MDX_ERR_STATE, "mdx_unet_create: no field data on the device");
    mdx_unet_opts_t o;
    if (opts) o = *opts;
    else mdx_default_unet_opts(&o);
    if (o.channels0 != 16 || (o.channels != 16 && o.channels != 32))
        return mdx_fail(ctx, MDX_ERR_ARG, "unet channels must be 16 and 16|32");
    if (o.extra_bottleneck < 0 || o.extra_bottleneck > MAX_EXTRA || o.capacity < 0 || !(o.slope > 0.0) || o.slope > 1.0 ||
        o.step_rule < 0 || o.step_rule > 1 || o.gate_period < 0)
        return mdx_fail(ctx, MDX_ERR_ARG, "unet options out of range");
    const mdx_dims& d = ctx->d;
    if (d.nx % 8 || d.ny % 8 || d.nz % 8) return mdx_fail(ctx, MDX_ERR_ARG, "unet needs nx, ny, nz multiples of 8");
    if (!ctx->bc.is_periodic[0] || !ctx->bc.is_periodic[2])
        return mdx_fail(ctx, MDX_ERR_ARG, "unet needs periodic x and z");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    mdx_unet_free(ctx);
    mdx_unet* U = new mdx_unet();
    ctx->unet = U;
    U->o = o;
    U->c0 = o.channels0;
    U->c1 = o.channels;
    U->pery = ctx->bc.is_periodic[1] ? 1 : 0;
    for (int l = 0; l < 4; ++l) U->L[l] = lvl{d.nx >> l, d.ny >> l, d.nz >> l, (long long)(d.nx >> l) * (d.ny >> l) * (d.nz >> l)};
    const int c0 = U->c0, c1 = U->c1;
    auto add = [&](int cin, int cout, int level) {
        conv_layer c;
        c.cin = cin;
        c.cout = cout;
        c.level = level;
        c.w_off = U->nparam;
        U->nparam += 27LL * cin * cout;
        c.b_off = U->nparam;
        U->nparam += cout;
        U->conv.push_back(c);
    };
    add(C_IN, c0, 0);
    add(c0, c0, 0);
    add(c0, c1, 1);
    add(c1, c1, 1);
    add(c1, c1, 2);
    add(c1, c1, 2);
    add(c1, c1, 3);
    add(c1, c1, 3);
    for (int e = 0; e < o.extra_bottleneck; ++e) add(c1, c1, 3);
    add(c1, c1, 2);   // dec2
    add(c1, c0, 1);   // dec1
    add(c0, c0, 0);   // dec0
    U->head_off = U->nparam;
    U->nparam += c0 + 1;
    int rc = alloc_net(ctx, U);
    if (rc != MDX_OK) {
        mdx_unet_free(ctx);
        return rc;
    }
    // He-uniform weights (fan-in 27*cin; the zero-padded input channels
    // count as NIN), zero biases, a small head
    std::vector<float> h((size_t)U->nparam, 0.f);
    uint64_t st = o.seed;
    for (auto& c : U->conv) {
        const int fan = 27 * (c.cin == C_IN && &c == &U->conv[0] ? NIN : c.cin);
        const double a = std::sqrt(6.0 / fan);
        for (long long i = 0; i < 27LL * c.cin * c.cout; ++i) {
            const int ci = (int)(i % c.cin);
            float v = (float)((2.0 * uniform01(st) - 1.0) * a);
            if (&c == &U->conv[0] && ci >= NIN) v = 0.f;
            h[(size_t)(c.w_off + i)] = v;
        }
    }
    for (int i = 0; i < c0; ++i) h[(size_t)(U->head_off + i)] = (float)((2.0 * uniform01(st) - 1.0) * std::sqrt(3.0 / c0));
    U->order_state = o.seed ^ 0x5DEECE66Dull;
    rc = mdx_unet_set_params(ctx, h.data(), U->nparam);
    if (rc != MDX_OK) {
        mdx_unet_free(ctx);
        return rc;
    }
    U->trained = false;
    return MDX_OK;
}

int mdx_unet_destroy(mdx_ctx_t* ctx) {
    if (!ctx) return mdx_fail(nullptr, MDX_ERR_ARG, "null context");
    cudaSetDevice(ctx->device);
    mdx_unet_free(ctx);
    return MDX_OK;
}

int mdx_unet_record(mdx_ctx_t* ctx, int on) {
    MDX_TRY(need_unet(ctx));
    static_cast<mdx_unet*>(ctx->unet)->recording = on != 0;
    return MDX_OK;
}

long long mdx_unet_param_count(const mdx_ctx_t* ctx) {
    if (!ctx || !ctx->unet) return 0;
    return static_cast<const mdx_unet*>(ctx->unet)->nparam;
}

int mdx_unet_get_params(mdx_ctx_t* ctx, float* host, long long n) {
    MDX_TRY(need_unet(ctx));
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (!host || n != U->nparam) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_unet_get_params: need %lld floats", U->nparam);
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    MDX_CUDA(ctx, cudaMemcpyAsync(host, U->param, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MDX_OK;
}

int mdx_unet_set_params(mdx_ctx_t* ctx, const float* host, long long n) {
    MDX_TRY(need_unet(ctx));
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (!host || n != U->nparam) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_unet_set_params: need %lld floats", U->nparam);
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    MDX_CUDA(ctx, cudaMemcpyAsync(U->param, host, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    MDX_TRY(export_weights(ctx, U));
    MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    U->trained = true;
    U->adam_t = 0;
    MDX_CUDA(ctx, cudaMemsetAsync(U->adam_m, 0, sizeof(float) * U->nparam, ctx->stream));
    MDX_CUDA(ctx, cudaMemsetAsync(U->adam_v, 0, sizeof(float) * U->nparam, ctx->stream));
    return MDX_OK;
}

int mdx_unet_get_out_scale(mdx_ctx_t* ctx, double* scale) {
    MDX_TRY(need_unet(ctx));
    if (!scale) return mdx_fail(ctx, MDX_ERR_ARG, "null argument");
    *scale = static_cast<mdx_unet*>(ctx->unet)->out_scale;
    return MDX_OK;
}

int mdx_unet_set_out_scale(mdx_ctx_t* ctx, double scale) {
    MDX_TRY(need_unet(ctx));
    if (!(scale > 0.0) || !std::isfinite(scale)) return mdx_fail(ctx, MDX_ERR_ARG, "out scale must be positive");
    static_cast<mdx_unet*>(ctx->unet)->out_scale = scale;
    return MDX_OK;
}

int mdx_unet_loss_grad(mdx_ctx_t* ctx, const float* in4, const float* target, double* loss, float* grad, float* out) {
    MDX_TRY(need_unet(ctx));
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (!in4 || !target) return mdx_fail(ctx, MDX_ERR_ARG, "null argument");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    const long long n = U->L[0].n;
    float* t = U->raw;   // scratch for the target
    MDX_CUDA(ctx, cudaMemcpyAsync(U->in, in4, sizeof(float) * NIN * n, cudaMemcpyHostToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemcpyAsync(t, target, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    MDX_CUDA(ctx, cudaMemsetAsync(U->grad, 0, sizeof(float) * U->nparam, ctx->stream));
    float* dout = nullptr;
    if (out) MDX_TRY(dalloc(ctx, &dout, n));
    int rc = loss_grad(ctx, U, U->in, t, 1.0f, dout);
    float sse = 0.f;
    if (rc == MDX_OK) {
        cudaMemcpyAsync(&sse, U->out + head_len<16>() - 1, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
        if (grad) cudaMemcpyAsync(grad, U->grad, sizeof(float) * U->nparam, cudaMemcpyDeviceToHost, ctx->stream);
        if (out) cudaMemcpyAsync(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream);
        const cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = mdx_fail(ctx, MDX_ERR_CUDA, "unet loss/grad: %s", cudaGetErrorString(e));
    }
    if (dout) cudaFree(dout);
    if (loss) *loss = (double)sse / (double)n;
    if (rc == MDX_OK) rc = check_tc(ctx, U);
    return rc;
}

int mdx_unet_train(mdx_ctx_t* ctx, int iters, double lr, double* loss_first, double* loss_last) {
    MDX_TRY(need_unet(ctx));
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    if (iters < 0 || !(lr > 0.0)) return mdx_fail(ctx, MDX_ERR_ARG, "mdx_unet_train: bad iters or lr");
    if (U->stored == 0) return mdx_fail(ctx, MDX_ERR_STATE, "mdx_unet_train: no snapshots recorded");
    MDX_CUDA(ctx, cudaSetDevice(ctx->device));
    const long long n = U->L[0].n;
    const long long stride = (NIN + 1) * n;
    // output scale: RMS of the stored targets
    {
        double acc = 0.0;
        for (int sl = 0; sl < U->stored; ++sl) {
            MDX_LAUNCH(ctx, MDX_T_OTHER, "unet target rms", k_sumsq, U->red_blocks, 256, 0, n,
                       U->snap + sl * stride + NIN * n, U->red_part);
            double a = 0.0;
            MDX_TRY(pairs_to_host(ctx, U, U->red_blocks, &a, nullptr));
            acc += a;
        }
        const double rms = std::sqrt(acc / ((double)n * U->stored));
        if (rms > 0.0 && std::isfinite(rms)) U->out_scale = rms;
    }
    const float tscale = (float)(1.0 / U->out_scale);
    MDX_CUDA(ctx, cudaEventRecord(U->ev[0], ctx->stream));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float sse_first = 0.f, sse_last = 0.f;
    std::vector<int> order;
    for (int it = 0; it < iters; ++it) {
        if (order.empty()) {   // a fresh seeded permutation of the stored snapshots
            order.resize(U->stored);
            for (int i = 0; i < U->stored; ++i) order[i] = i;
            for (int i = U->stored - 1; i > 0; --i) std::swap(order[i], order[splitmix(U->order_state) % (uint64_t)(i + 1)]);
        }
        const int sl = order.back();
        order.pop_back();
        const float* in4 = U->snap + sl * stride;
        MDX_TRY(loss_grad(ctx, U, in4, in4 + NIN * n, tscale, nullptr));
        U->adam_t++;
        const float c1 = 1.f / (1.f - std::pow(b1, (float)U->adam_t));
        const float c2 = 1.f / (1.f - std::pow(b2, (float)U->adam_t));
        MDX_LAUNCH(ctx, MDX_T_OTHER, "unet adam", k_adam, nblocks(U->nparam), 256, 0, U->nparam, U->param, U->grad,
                   U->adam_m, U->adam_v, (float)lr, b1, b2, eps, c1, c2);
        MDX_TRY(export_weights(ctx, U));
        if (it == 0 || it == iters - 1) {
            float sse = 0.f;
            MDX_CUDA(ctx, cudaMemcpyAsync(&sse, U->out + head_len<16>() - 1, sizeof(float), cudaMemcpyDeviceToHost,
                                          ctx->stream));
            MDX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (it == 0) sse_first = sse;
            sse_last = sse;
        }
    }
    MDX_CUDA(ctx, cudaEventRecord(U->ev[1], ctx->stream));
    MDX_CUDA(ctx, cudaEventSynchronize(U->ev[1]));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, U->ev[0], U->ev[1]) == cudaSuccess) U->st.train_ms = ms;
    MDX_TRY(check_tc(ctx, U));
    U->trained = true;
    if (loss_first) *loss_first = (double)sse_first / (double)n;
    if (loss_last) *loss_last = (double)sse_last / (double)n;
    return MDX_OK;
}

int mdx_unet_stats(mdx_ctx_t* ctx, mdx_unet_stats_t* out) {
    MDX_TRY(need_unet(ctx));
    if (!out) return mdx_fail(ctx, MDX_ERR_ARG, "null argument");
    mdx_unet* U = static_cast<mdx_unet*>(ctx->unet);
    U->st.snapshots = U->total_snaps;
    U->st.stored = U->stored;
    U->st.trained = U->trained ? 1 : 0;
    U->st.out_scale = U->out_scale;
    *out = U->st;
    return MDX_OK;
}

}  // extern "C"
