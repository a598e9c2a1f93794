// FR P=3 stage kernels for sm_100a.
//
// One SSP-RK3 stage of the reference (src/solver.rs:262-317) is a volume
// kernel, three face kernels (+ the y-wall kernel) and an RK kernel
// (src/cuda/rhs.cu:344-739, src/cuda/rk.cu:85-115): seven passes over HBM
// with 6 gradient-slice and 6 face-correction arrays in between. Here a
// stage is two element-local kernels.
//
// Phase A — 16 threads per element; in the pass of direction d each thread
// owns the d-line through face point l (l = j+4k for x, i+4k for y, i+4j for
// z, the reference's face-point numbering), so 1-D operators act on four
// registers:
//   P1  the element state (x-lines, 128-bit loads) -> smem; each thread
//        keeps its own x-line for the x pass
//   P2-4 per direction (x, y, then z after a barrier): own and neighbour
//        face values (BR1 common solution, slip-wall mirror
//        rhs.cu:111-114), corrected gradient along the line
//        (rhs.cu:373-461); at the minus face of the line the interface flux
//        F_I is solved once for both sides (j = F_I - Fe_own here, F_I kept
//        in registers); at the plus face j = -Fe_own (slip wall:
//        j = [0,0,p_w,0,0] - Fe, complete). The y neighbours' traces come
//        from one 128-bit load per variable and side and a lane
//        reduce-scatter; the z pass also does P5 for the z faces.
//   P5  x / y faces: gradient at the face (11 components), own viscous
//        flux Fv; j += 1/2 Fv_own; to the face buffer for the neighbours:
//        F_I - 1/2 Fv_own at the minus faces (all the minus neighbour still
//        needs at its plus face), Fv_own at the plus faces
//   P6  x-threads: pointwise Euler - viscous fluxes of their 4 points
//        (rhs.cu:229-266); F_y, F_z -> smem, the x-divergence of the
//        thread's own x-line accumulated in registers
//   P7  x-threads: divergence of F_y / F_z at their 4 points from the
//        x-lines of their k-plane / j-column (128-bit loads)
//   P8  x-threads: RHS = -div + forcing (rhs.cu:505-509), lifting
//        -(j_L g_L' + j_R g_R') jac (rk.cu:12-25), RK combination
//        a*u0 + b*u + c*(RHS + lift) (rk.cu:27-83), 128-bit stores.
//   The face correction of the reference, j = F_I - 1/2(Fv_L + Fv_R) -
//   (Fe_own - Fv_own), is then complete except for the terms that belong to
//   the neighbour: F_I at the plus faces and -1/2 Fv_nbr at every non-wall
//   face.
// Phase B — reads those from the face buffer records of the +x/+y/+z
// neighbours (F_I - 1/2 Fv_nbr) and -x/-y/-z neighbours (Fv_nbr) and adds
// their lifted contribution. With an f32 state
// phase A stores the unrounded RHS instead of the new state and phase B
// performs the RK combination, so the state is rounded once per stage:
// phase B's increments are often below half an f32 ulp of E and rho*u, and
// rounding the state before adding them would drop them systematically.
// Phase B always runs (the plus-face F_I comes from the neighbour even when
// mu == 0).
//
// Types: S = stored state, P = state arithmetic (face values, pressure
// recovery, RK accumulation), C = flux arithmetic. Reference-compatible
// pipelines use P == C; the mixed-precision form uses S = P = double with
// C = float.
#pragma once

#include <cuda_bf16.h>

#include "od_launch.h"
#include "od_physics.cuh"

namespace od {

constexpr int NP = 4;   // points per direction
constexpr int NF = 16;  // points per face
constexpr int NE = 64;  // points per element
constexpr int NV = 5;   // conserved variables
constexpr int LPE = 16; // threads (lines) per element

template <class T>
struct Tab {
    T D[16];   // D[a*4+m] = l'_m(x_a)
    T eL[4];   // l_m(-1)
    T eR[4];   // l_m(+1)
    T gL[4];   // Radau g_L'(x_a)
    T gR[4];   // Radau g_R'(x_a)
};

// The operators of each direction scaled by its Jacobian 2/h, so that the
// corrected gradient, the divergence and the lifting are pure FMA chains:
// d[dir][a*4+m] = D[a*4+m] jac[dir], gl / gr[dir][a] = g_L' / g_R'(x_a) jac[dir]
// (products rounded in T).
template <class T>
struct ScaledTab {
    T d[3][16];
    T gl[3][4];
    T gr[3][4];
};

template <class T, class TabT>
__host__ ScaledTab<T> scale_tab(const TabT& t, const T* jac) {
    ScaledTab<T> r;
    for (int dir = 0; dir < 3; ++dir) {
        for (int i = 0; i < 16; ++i) r.d[dir][i] = (T)(t.D[i] * jac[dir]);
        for (int a = 0; a < 4; ++a) {
            r.gl[dir][a] = (T)(t.gL[a] * jac[dir]);
            r.gr[dir][a] = (T)(t.gR[a] * jac[dir]);
        }
    }
    return r;
}

// Division of a 32-bit unsigned value by a divisor fixed for the launch: a
// multiply-high and two shifts instead of the integer division sequence
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, section 4): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, n / d = (t + ((n - t) >> min(l, 1))) >>
// max(l - 1, 0) where t = mulhi(m, n), for every n and d in [1, 2^32).
struct FastDiv {
    unsigned m, s1, s2;
};

__host__ inline FastDiv make_fastdiv(unsigned d) {
    unsigned l = 0;
    while (l < 32 && (1ull << l) < d) ++l;
    FastDiv f;
    f.m = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
    f.s1 = l < 1 ? l : 1;
    f.s2 = l > 0 ? l - 1 : 0;
    return f;
}

__device__ __forceinline__ unsigned fast_div(unsigned n, const FastDiv& f) {
    const unsigned t = __umulhi(f.m, n);
    return (t + ((n - t) >> f.s1)) >> f.s2;
}

// Element indices are below 2^31 (od_create rejects larger meshes).
struct Mesh {
    int nx, ny, nz, y_wall;
    long long nelem, npts;
    FastDiv fx, fy;   // division by nx and by ny
};

__host__ inline void mesh_set_div(Mesh& m) {
    m.fx = make_fastdiv((unsigned)m.nx);
    m.fy = make_fastdiv((unsigned)m.ny);
}

// (ex, ey, ez) of element e = ex + nx (ey + ny ez)
__device__ __forceinline__ void elem_coords(const Mesh& m, long long e, int& ex, int& ey, int& ez) {
    const unsigned u = (unsigned)e;
    const unsigned q = fast_div(u, m.fx);
    const unsigned q2 = fast_div(q, m.fy);
    ex = (int)(u - q * (unsigned)m.nx);
    ey = (int)(q - q2 * (unsigned)m.ny);
    ez = (int)q2;
}

// point index inside an element: i + 4 j + 16 k
__device__ __forceinline__ constexpr int pid(int i, int j, int k) { return i + NP * j + NF * k; }

// point m of the direction-D line through face point fp
template <int D>
__device__ __forceinline__ int line_pt(int fp, int m) {
    if constexpr (D == 0) return m + NP * fp;                  // fp = j + 4k
    else if constexpr (D == 1) return (fp & 3) + NP * m + NF * (fp >> 2);  // fp = i + 4k
    else return fp + NF * m;                                   // fp = i + 4j
}

// Face value from the four samples of a line; one fixed FMA chain so that the
// two elements sharing a face compute bit-identical face states.
template <class T, class CC>
__device__ __forceinline__ T trace4(const T* q, const CC& c) {
    return fma(q[3], c[3], fma(q[2], c[2], fma(q[1], c[1], q[0] * c[0])));
}

// Face values at both ends of a line (trace4 with cL and with cR).
template <class T, class CL, class CR>
__device__ __forceinline__ void trace4_lr(const T* q, const CL& cL, const CR& cR, T& oL, T& oR) {
    oL = trace4(q, cL);
    oR = trace4(q, cR);
}

// r[a] = sum_m D[a*4+m] q[m] for a = 0..3 (the FR derivative along a line,
// D already scaled by the Jacobian). Paired f32 forms (FFMA2) of these loops
// measured 3% slower on B200: the pairs cost operand moves and registers.
template <class T, class DM>
__device__ __forceinline__ void deriv4(const T* q, const DM& D, T* r) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        T df = D[a * 4] * q[0];
#pragma unroll
        for (int mm = 1; mm < 4; ++mm) df = fma(D[a * 4 + mm], q[mm], df);
        r[a] = df;
    }
}

// Sum over the four lanes of an aligned lane group (4g .. 4g+3) of p[q], for
// lane q = lane & 3 of the group: a reduce-scatter in two shuffle rounds
// (partner lane ^ 2 for the pair of components a lane keeps, then lane ^ 1).
// Every lane forms (p_q + p_q^2) + (p_q^1 + p_q^3), which by commutativity is
// the same value, (p_0 + p_2) + (p_1 + p_3), for all four. All 32 lanes of
// the warp must call it together.
template <class T>
__device__ __forceinline__ T sum4_scatter(const T (&p)[4], int q) {
    const bool hi = (q & 2) != 0;
    const T a0 = hi ? p[2] : p[0], a1 = hi ? p[3] : p[1];
    const T b0 = hi ? p[0] : p[2], b1 = hi ? p[1] : p[3];
    const T c0 = a0 + __shfl_xor_sync(0xffffffffu, b0, 2);
    const T c1 = a1 + __shfl_xor_sync(0xffffffffu, b1, 2);
    const bool odd = (q & 1) != 0;
    const T d = odd ? c1 : c0, e = odd ? c0 : c1;
    return d + __shfl_xor_sync(0xffffffffu, e, 1);
}

// neighbour across face (d, side) or -1 for a slip wall
__device__ __forceinline__ long long neighbour(const Mesh& m, int ex, int ey, int ez, int d, int side) {
    int c0 = ex, c1 = ey, c2 = ez;
    if (d == 0) {
        c0 += side ? 1 : -1;
        c0 = c0 < 0 ? c0 + m.nx : (c0 >= m.nx ? c0 - m.nx : c0);
    } else if (d == 1) {
        c1 += side ? 1 : -1;
        if (m.y_wall && (c1 < 0 || c1 >= m.ny)) return -1;
        c1 = c1 < 0 ? c1 + m.ny : (c1 >= m.ny ? c1 - m.ny : c1);
    } else {
        c2 += side ? 1 : -1;
        c2 = c2 < 0 ? c2 + m.nz : (c2 >= m.nz ? c2 - m.nz : c2);
    }
    return (long long)(c0 + m.nx * (c1 + m.ny * c2));
}

// ---- 4-wide loads / stores (16-byte aligned for float, 32-byte for double)
template <class T>
__device__ __forceinline__ void ld4s(const T* p, T* q) {
    if constexpr (sizeof(T) == 4) {
        float4 v = *reinterpret_cast<const float4*>(p);
        q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
    } else {
        double2 a = reinterpret_cast<const double2*>(p)[0];
        double2 b = reinterpret_cast<const double2*>(p)[1];
        q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y;
    }
}

template <class T>
__device__ __forceinline__ void st4s(T* p, const T* q) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(q[0], q[1], q[2], q[3]);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2(q[0], q[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(q[2], q[3]);
    }
}

// global 4-wide load of S values converted to P (read-only path)
template <class S, class P>
__device__ __forceinline__ void ldg4(const S* __restrict__ p, P* q) {
    if constexpr (sizeof(S) == 4) {
        float4 v = __ldg(reinterpret_cast<const float4*>(p));
        q[0] = (P)v.x; q[1] = (P)v.y; q[2] = (P)v.z; q[3] = (P)v.w;
    } else {
        double2 a = __ldg(reinterpret_cast<const double2*>(p));
        double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        q[0] = (P)a.x; q[1] = (P)a.y; q[2] = (P)b.x; q[3] = (P)b.y;
    }
}

// coherent 4-wide load (for data the same kernel later overwrites)
template <class S, class P>
__device__ __forceinline__ void ldc4(const S* p, P* q) {
    S w[4];
    ld4s(p, w);
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = (P)w[a];
}

template <class S, class P>
__device__ __forceinline__ void stg4(S* p, const P* q) {
    if constexpr (sizeof(S) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
    } else {
        reinterpret_cast<double2*>(p)[0] = make_double2((double)q[0], (double)q[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2((double)q[2], (double)q[3]);
    }
}

// gradient components the direction-D viscous flux reads
// (x omits 8,10,13,14; y omits 5,9,12,14; z omits 4,6,12,13 — rhs.cu:129,151,169)
template <int D>
__device__ __forceinline__ constexpr bool grad_used(int c) {
    constexpr unsigned omit = D == 0 ? ((1u << 8) | (1u << 10) | (1u << 13) | (1u << 14))
                            : D == 1 ? ((1u << 5) | (1u << 9) | (1u << 12) | (1u << 14))
                                     : ((1u << 4) | (1u << 6) | (1u << 12) | (1u << 13));
    return !((omit >> c) & 1u);
}

// Shared-memory slot of one element in phase A.
// ---- shared-memory point layout
// Points of an element are stored at p ^ (((p >> 3) & 4) | par << 3): the
// j index is XOR-swizzled with bit 1 of k and with the element's parity
// inside its warp (two elements per warp), and every element slot is a
// multiple of 32 words plus 16. With these, the three access patterns of a
// half-warp (16 x-lines as 128-bit vectors, 16 y-lines and 16 z-lines as
// scalars) hit 32 distinct banks across the whole warp.
__device__ __forceinline__ int sw(int p, int swz) { return p ^ (((p >> 3) & 4) | swz); }

template <class P, class C>
struct SlotBytes {
    static constexpr int base = 15 * NE * (int)sizeof(C) + NV * NE * (int)sizeof(P) + 4 * NV * NF * (int)sizeof(C);
    static constexpr int words = base / 4;
    static constexpr int pad_words = ((16 - words % 32) + 32) % 32 == 0 ? 32 : ((16 - words % 32) + 32) % 32;
};

// Shared-memory slot of one element in phase A.
template <class P, class C>
struct alignas(16) SlotA {
    C g[15][NE];          // gradient; P6: F_y rows 0-4, F_z rows 5-9
    P u[NV][NE];          // state
    C j[4][NV][NF];       // y / z face corrections without -1/2 Fv_nbr [face - 2][var][face pt]; the x faces of
                          // a line belong to its own thread and stay in registers
    float pad[SlotBytes<P, C>::pad_words];
};

template <class S, class P, class C>
struct StageAParams {
    using S_t = S;
    using P_t = P;
    using C_t = C;
    const S* u_in;
    const S* u0;
    S* u_out;       // new state, or the RHS when phase B performs the RK combination
    C* fv;          // [elem][dir 3][var 4][face pt 16]: own viscous flux (components 1..4) at the plus faces
    C* fi;          // [elem][dir 3][var 5][face pt 16]: F_I - 1/2 Fv_own at the minus faces
    Mesh m;
    Tab<P> tp;
    Tab<C> tc;
    ScaledTab<C> sc;
    C jac[3];
    P ra, rb, rc;
    C mu, forcing;
    C suth;             // Sutherland S = s_suth / t_ref, < 0: constant mu
    C kappa;            // heat-flux coefficient of the constant mu (heat_coeff_host)
    int flags;
    int flux;           // scheme id, read when the kernel's FLUX is kFluxRuntime
    long long e0, e1;   // element range of this launch
    StageFeatures feat; // the closure's features, written by the FEAT kernels (f32)
};


// P1b of phase A with the closure attached: the features of the element's
// input state at the thread's four points (the same operations, in the same
// order, as the closure's features kernel: x derivatives from the thread's
// x-line, y / z derivatives from the x-lines of its k-plane / j-column),
// staged as bf16 in the gradient rows (not written before P2) and stored in
// the fused inference kernel's tile layout as 16-byte chunks.
template <class PA, class P = typename PA::P_t, class C = typename PA::C_t>
__device__ __forceinline__ void stage_a_features(const PA& A, SlotA<P, C>& sm, long long e, int l, int swz,
                                                 bool live, const P (&qx)[NV][4]) {
    const StageFeatures& fp = A.feat;
    const int j = l & 3, k = l >> 2;
    float d[4][3][4];   // [var][direction][point of the line]
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        float ly[4][4], lz[4][4];   // the x-lines (m, k) and (j, m), m = 0..3
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            ld4s(&sm.u[v][sw(4 * (m + 4 * k), swz)], ly[m]);
            ld4s(&sm.u[v][sw(4 * (j + 4 * m), swz)], lz[m]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                sx += fp.D[i * 4 + m] * qx[v][m];
                sy += fp.D[j * 4 + m] * ly[m][i];
                sz += fp.D[k * 4 + m] * lz[m][i];
            }
            d[v][0][i] = sx * fp.jac[0];
            d[v][1][i] = sy * fp.jac[1];
            d[v][2][i] = sz * fp.jac[2];
        }
    }
    __nv_bfloat16* st = reinterpret_cast<__nv_bfloat16*>(&sm.g[0][0]);   // [channel][64 points]
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int p = i + 4 * l;
        const float ir = 1.0f / qx[0][i];
        float ch[kFeatChan];
#pragma unroll
        for (int v = 0; v < 5; ++v) ch[v] = qx[v][i];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ch[5 + 3 * a + b] = (d[1 + a][b][i] - qx[1 + a][i] * ir * d[0][b][i]) * ir;
#pragma unroll
        for (int c = 0; c < kFeatChan; ++c)
            st[c * 64 + p] =
                __float2bfloat16_rn(fminf(fmaxf((ch[c] - fp.mean[c]) * fp.inv_scale[c], -kFeatClip), kFeatClip));
    }
    __syncthreads();
    if (live) {
        // tile (e / 128), channel c: a 128 x 64 block, row e % 128, 16-byte
        // chunk kc at ((row / 8) * 1024 + kc * 128 + (row % 8) * 16) bytes
        char* tile = reinterpret_cast<char*>(fp.X) + (size_t)(e >> 7) * (128 * 64 * 2 * kFeatChan);
        const int r = (int)(e & 127);
        for (int q8 = l; q8 < kFeatChan * 8; q8 += 16) {
            const int c = q8 >> 3, kc = q8 & 7;
            *reinterpret_cast<uint4*>(tile + (size_t)c * (128 * 64 * 2) + (r >> 3) * 1024 + kc * 128 + (r & 7) * 16) =
                *reinterpret_cast<const uint4*>(&st[c * 64 + 8 * kc]);
        }
    }
    __syncthreads();   // the gradient rows are P2's from here
}

// Inviscid part of the face corrections at the two faces of a line. Each
// face's interface flux F_I is solved once, by the element on its plus side
// (the face is that element's minus face): there j = F_I - Fe_own and F_I is
// stored for the neighbour; on the element's plus face j = -Fe_own here and
// phase B adds the neighbour's F_I. Slip walls (rhs.cu:311-339) are complete
// here: j = [0, 0, p_wall, 0, 0] - Fe_own with p_wall from the own flux.
template <class M, int D, class P, class C>
__device__ __forceinline__ void wall_face(const FaceState<C>& so, const C* fe, C* j) {
    const C pw = fe[2] - so.q[2] * so.q[2] * so.ir;
#pragma unroll
    for (int v = 0; v < NV; ++v) j[v] = -fe[v];
    j[2] = pw - fe[2];
}

// so: the own face state (make_face_state of the own face values).
template <class M, int FLUX, int D, class P, class C>
__device__ __forceinline__ void minus_face(const FaceState<C>& so, const P* nbr, bool wall, C* j, C* fi, int rflux) {
    C fe[NV];
    euler_flux<D>(so, fe);
    if (wall) {
        wall_face<M, D, P, C>(so, fe, j);
        return;
    }
    C praw;
    FaceState<C> sn = make_face_state<M, C, P>(nbr, praw);
    if constexpr (FLUX == kFluxRuntime)
        interface_flux_rt<M, D>(rflux, sn, so, fi);
    else
        interface_flux<M, FLUX, D>(sn, so, fi);
#pragma unroll
    for (int v = 0; v < NV; ++v) j[v] = fi[v] - fe[v];
}

template <class M, int D, class P, class C>
__device__ __forceinline__ void plus_face(const FaceState<C>& so, bool wall, C* j) {
    C fe[NV];
    euler_flux<D>(so, fe);
    if (wall) {
        wall_face<M, D, P, C>(so, fe, j);
        return;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) j[v] = -fe[v];
}

// Swizzled row offsets of the three lines of thread l, computed once per
// tile: x-line start, the four y-line points and the two z-line bases
// (points mm < 2 and mm >= 2, + 16 mm).
struct LineIdx {
    int x;
    int y[4];
    int z[2];
};

__device__ __forceinline__ LineIdx line_idx(int l, int swz) {
    LineIdx li;
    li.x = sw(4 * l, swz);
#pragma unroll
    for (int mm = 0; mm < 4; ++mm) li.y[mm] = sw(line_pt<1>(l, mm), swz);
    li.z[0] = sw(line_pt<2>(l, 0), swz);
    li.z[1] = sw(line_pt<2>(l, 2), swz) - 32;
    return li;
}

template <int D>
__device__ __forceinline__ int line_off(const LineIdx& li, int mm) {
    if constexpr (D == 1) return li.y[mm];
    else return li.z[mm >> 1] + 16 * mm;
}

// load / store the 4 samples of the thread's direction-D line of a swizzled row
template <int D, class T>
__device__ __forceinline__ void row_line_load(const T* row, const LineIdx& li, T* w) {
    if constexpr (D == 0) {
        ld4s(row + li.x, w);
    } else {
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) w[mm] = row[line_off<D>(li, mm)];
    }
}

template <int D, class T>
__device__ __forceinline__ void row_line_store(T* row, const LineIdx& li, const T* w) {
    if constexpr (D == 0) {
        st4s(row + li.x, w);
    } else {
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) row[line_off<D>(li, mm)] = w[mm];
    }
}

// Viscous part at one face point: j += 1/2 Fv_own; to the face buffer for
// the neighbour's phase B: F_I - 1/2 Fv_own at a minus face (fi: the
// interface flux solved in the line pass), Fv_own (components 1..4) at a
// plus face.
// REG: the face's correction j is in registers (jreg), else in shared memory.
// s, praw: the face state (make_face_state of the face values).
template <class M, int D, bool REG, class PA, class P = typename PA::P_t, class C = typename PA::C_t>
__device__ __forceinline__ void viscous_face(const PA& A, SlotA<P, C>& sm, long long e, int l, int side,
                                             const FaceState<C>& s, C praw, const C* gt, bool live, C* jreg,
                                             const C* fi) {
    const int f = 2 * D + side;
    C fv[NV];
    const C mu = viscosity<M>(A.mu, A.suth, s);
    viscous_flux<D>(s, praw, gt, mu, heat_coeff<M>(mu, A.kappa), fv);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if constexpr (REG)
            jreg[v] += (C)0.5 * fv[v];
        else
            sm.j[f - 2][v][l] += (C)0.5 * fv[v];
    }
    if (!live) return;
    if (side == 0) {
        C* out = A.fi + ((e * 3 + D) * NV) * NF + l;
        out[0] = fi[0];
#pragma unroll
        for (int v = 1; v < NV; ++v) out[v * NF] = fi[v] - (C)0.5 * fv[v];
    } else {
        C* out = A.fv + ((e * 3 + D) * 4) * NF + l;
#pragma unroll
        for (int v = 1; v < NV; ++v) out[(v - 1) * NF] = fv[v];
    }
}

// P2-P4: one direction of the gradient / face-value pass for line l.
// qx: the thread's own x-line as P1 loaded it (used by the x pass instead of
// reading it back from shared memory). The z pass (the last one, run after
// the x and y gradients are in shared memory) also does the z faces' viscous
// part (P5 for z): its normal gradient components are traced from registers
// and the z-face corrections are stored once, complete.
template <class M, int FLUX, int D, class PA, class P = typename PA::P_t, class C = typename PA::C_t>
__device__ __forceinline__ void line_pass(const PA& A, SlotA<P, C>& sm, long long e, int l, const LineIdx& li,
                                          bool live, const long long nb0, const long long nb1, P* oL, P* oR,
                                          C (&jx)[2][NV], C* fi, const P (&qx)[NV][4]) {
    using S = typename PA::S_t;
    const Mesh& m = A.m;
    P q[NV][4];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if constexpr (D == 0) {
#pragma unroll
            for (int a = 0; a < 4; ++a) q[v][a] = qx[v][a];
        } else {
            row_line_load<D>(sm.u[v], li, q[v]);
        }
    }
    P nL[NV], nR[NV];
    if constexpr (D == 1) {
        // y neighbours: the neighbour's x-line l (points (0..3, j, k), j = l & 3,
        // k = l >> 2) in one 128-bit load per variable, weighted with the trace
        // coefficient of row j and summed over the four rows of the k-plane by
        // the four lanes that hold them, so that lane l ends with the trace at
        // face point (i, k) = (l & 3, l >> 2), its own y-line. Slip walls (no
        // neighbour) load nothing and mirror the own face value instead.
        const int q4 = l & 3;
        const P cm = A.tp.eR[q4], cp = A.tp.eL[q4];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            trace4_lr(q[v], A.tp.eL, A.tp.eR, oL[v], oR[v]);
            const P refl = (v > 0 && v < 4) ? (P)-1.0 : (P)1.0;
            P wm[4] = {(P)0, (P)0, (P)0, (P)0}, wp[4] = {(P)0, (P)0, (P)0, (P)0};
            if (nb0 >= 0) ldg4<S, P>(A.u_in + v * m.npts + nb0 * NE + 4 * l, wm);
            if (nb1 >= 0) ldg4<S, P>(A.u_in + v * m.npts + nb1 * NE + 4 * l, wp);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                wm[a] *= cm;
                wp[a] *= cp;
            }
            const P sL = sum4_scatter(wm, q4);
            const P sR = sum4_scatter(wp, q4);
            nL[v] = nb0 >= 0 ? sL : oL[v] * refl;
            nR[v] = nb1 >= 0 ? sR : oR[v] * refl;
        }
    } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        trace4_lr(q[v], A.tp.eL, A.tp.eR, oL[v], oR[v]);
        const P refl = (v > 0 && v < 4) ? (P)-1.0 : (P)1.0;
        if (D != 1 || nb0 >= 0) {   // only y can have walls: x and z neighbours always exist
            P w[4];
            const S* base = A.u_in + v * m.npts + nb0 * NE;
            if constexpr (D == 0) {
                ldg4<S, P>(base + 4 * l, w);
            } else {
#pragma unroll
                for (int mm = 0; mm < 4; ++mm) w[mm] = (P)__ldg(base + line_pt<D>(l, mm));
            }
            nL[v] = trace4(w, A.tp.eR);
        } else {
            nL[v] = oL[v] * refl;
        }
        if (D != 1 || nb1 >= 0) {
            P w[4];
            const S* base = A.u_in + v * m.npts + nb1 * NE;
            if constexpr (D == 0) {
                ldg4<S, P>(base + 4 * l, w);
            } else {
#pragma unroll
                for (int mm = 0; mm < 4; ++mm) w[mm] = (P)__ldg(base + line_pt<D>(l, mm));
            }
            nR[v] = trace4(w, A.tp.eL);
        } else {
            nR[v] = oR[v] * refl;
        }
    }
    }
    // corrected gradient along the line (BR1): jl g_L' + jr g_R' + D q, all
    // scaled by the Jacobian, as one FMA chain per point
    C gnL[NV], gnR[NV];   // z pass: face values of the normal gradient components
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const C jl = (C)((P)0.5 * (nL[v] + oL[v]) - oL[v]);
        const C jr = (C)((P)0.5 * (nR[v] + oR[v]) - oR[v]);
        C gv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            C gg = fma(jr, A.sc.gr[D][a], jl * A.sc.gl[D][a]);
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) gg = fma(A.sc.d[D][a * 4 + mm], (C)q[v][mm], gg);
            if constexpr (sizeof(C) == 8) {
                if (A.flags & kRoundQ) gg = (C)(float)gg;
            }
            gv[a] = gg;
        }
        row_line_store<D>(sm.g[3 * v + D], li, gv);
        if constexpr (D == 2) trace4_lr(gv, A.tc.eL, A.tc.eR, gnL[v], gnR[v]);
    }
    // inviscid parts at the two faces of this line; F_I stays in registers
    // until the minus face's viscous flux is known (P5)
    C j0[NV], j1[NV];
    C prawL, prawR;
    const FaceState<C> sL = make_face_state<M, C, P>(oL, prawL);
    const FaceState<C> sR = make_face_state<M, C, P>(oR, prawR);
    minus_face<M, FLUX, D, P, C>(sL, nL, D == 1 && nb0 < 0, j0, fi, A.flux);
    plus_face<M, D, P, C>(sR, D == 1 && nb1 < 0, j1);
    if constexpr (D == 2) {
        // z faces (never walls): the 11 gradient components the z flux reads,
        // the normal ones from registers, the x / y ones from shared memory
        C gL[15], gR[15];
#pragma unroll
        for (int c = 0; c < 15; ++c) {
            if (!grad_used<2>(c)) {
                gL[c] = (C)0;
                gR[c] = (C)0;
            } else if (c % 3 == 2) {
                gL[c] = gnL[c / 3];
                gR[c] = gnR[c / 3];
            } else {
                C w[4];
                row_line_load<2>(sm.g[c], li, w);
                trace4_lr(w, A.tc.eL, A.tc.eR, gL[c], gR[c]);
            }
        }
        viscous_face<M, 2, true>(A, sm, e, l, 0, sL, prawL, gL, live, j0, fi);
        viscous_face<M, 2, true>(A, sm, e, l, 1, sR, prawR, gR, live, j1, fi);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if constexpr (D == 0) {
            jx[0][v] = j0[v];
            jx[1][v] = j1[v];
        } else {
            sm.j[2 * D - 2][v][l] = j0[v];
            sm.j[2 * D - 1][v][l] = j1[v];
        }
    }
}

// The reference's y-face gradient slice multiplies with __fmul_rn, a float
// intrinsic, also in its f64 build (rhs.cu:145-160): products and pair sums
// in f32. Reproduced on request (kRefYSlice) for bit-level drop-in parity.
template <class C, class CC>
__device__ __forceinline__ C ref_y_slice(const C* w, const CC& c) {
    const float a = __fadd_rn(__fmul_rn((float)w[0], (float)c[0]), __fmul_rn((float)w[1], (float)c[1]));
    const float b = __fadd_rn(__fmul_rn((float)w[2], (float)c[2]), __fmul_rn((float)w[3], (float)c[3]));
    return (C)__fadd_rn(a, b);
}

// P5: face values and face gradient along the D-line of thread l, viscous
// flux at both faces of the line.
template <class M, int D, class PA, class P = typename PA::P_t, class C = typename PA::C_t>
__device__ __forceinline__ void face_grad_pass(const PA& A, SlotA<P, C>& sm, long long e, int l,
                                               const LineIdx& li, bool wall0, bool wall1, bool live, const P* tL,
                                               const P* tR, C (&jx)[2][NV], const C* fi) {
    if (wall0 && wall1) return;
    C gL[15], gR[15];
    const bool ref_y = D == 1 && sizeof(C) == 8 && (A.flags & kRefYSlice);
#pragma unroll
    for (int c = 0; c < 15; ++c) {
        if (!grad_used<D>(c)) {
            gL[c] = (C)0;
            gR[c] = (C)0;
            continue;
        }
        C w[4];
        row_line_load<D>(sm.g[c], li, w);
        if (ref_y) {
            gL[c] = ref_y_slice(w, A.tc.eL);
            gR[c] = ref_y_slice(w, A.tc.eR);
        } else {
            trace4_lr(w, A.tc.eL, A.tc.eR, gL[c], gR[c]);
        }
    }
    // face values: kept in registers from the line pass (f32), else recomputed
    P qL[NV], qR[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if constexpr (sizeof(P) == 4) {
            qL[v] = tL[v];
            qR[v] = tR[v];
        } else {
            P w[4];
            row_line_load<D>(sm.u[v], li, w);
            trace4_lr(w, A.tp.eL, A.tp.eR, qL[v], qR[v]);
        }
    }
    if (!wall0) {
        C praw;
        const FaceState<C> st = make_face_state<M, C, P>(qL, praw);
        viscous_face<M, D, D == 0>(A, sm, e, l, 0, st, praw, gL, live, jx[0], fi);
    }
    if (!wall1) {
        C praw;
        const FaceState<C> st = make_face_state<M, C, P>(qR, praw);
        viscous_face<M, D, D == 0>(A, sm, e, l, 1, st, praw, gR, live, jx[1], fi);
    }
}

// P7 + P8 of phase A for one live element: the y / z divergences of the
// x-line's four points, RHS = -div + forcing, own-face lifting
// -(j_L g_L' + j_R g_R') jac, then the RK combination, or (deferred RK) the
// unrounded RHS + own lift for phase B.
// The y derivative at (i, j, k) reads F_y at (i, 0..3, k): the four x-lines of
// the thread's k-plane; the z derivative reads F_z at (i, j, 0..3): the four
// x-lines of its j-column. Each is one 128-bit shared load per x-line (lanes
// of the same plane / column load the same line: broadcasts), so no pass
// along y and z lines and no barrier before the update. Operation order per
// point as a derivative along the line: D[a][0] F_0, then FMAs for m = 1..3.
template <class PA, class P = typename PA::P_t, class C = typename PA::C_t>
__device__ __forceinline__ void stage_a_update(const PA& A, SlotA<P, C>& sm, long long ec, int l, int swz,
                                               const C (&divx)[NV][4], const C (&jx)[2][NV]) {
    using S = typename PA::S_t;
    const Mesh& m = A.m;
    const int lj = l & 3, lk = l >> 2;   // this x-line's (j, k)
    const bool defer = (A.flags & kDeferRK) != 0;
    C cy[4], cz[4];   // derivative rows of this thread's j (y) and k (z)
#pragma unroll
    for (int mm = 0; mm < 4; ++mm) {
        cy[mm] = A.sc.d[1][lj * 4 + mm];
        cz[mm] = A.sc.d[2][lk * 4 + mm];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        C dy[4], dz[4], jy0[4], jy1[4], jz0[4], jz1[4];
        const C* dx = divx[v];
        {
            C f[4][4];
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) ld4s(&sm.g[v][sw(4 * (mm + 4 * lk), swz)], f[mm]);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                C d = cy[0] * f[0][i];
#pragma unroll
                for (int mm = 1; mm < 4; ++mm) d = fma(cy[mm], f[mm][i], d);
                dy[i] = d;
            }
        }
        {
            C f[4][4];
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) ld4s(&sm.g[5 + v][sw(4 * (lj + 4 * mm), swz)], f[mm]);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                C d = cz[0] * f[0][i];
#pragma unroll
                for (int mm = 1; mm < 4; ++mm) d = fma(cz[mm], f[mm][i], d);
                dz[i] = d;
            }
        }
        ld4s(&sm.j[0][v][4 * lk], jy0);
        ld4s(&sm.j[1][v][4 * lk], jy1);
        ld4s(&sm.j[2][v][4 * lj], jz0);
        ld4s(&sm.j[3][v][4 * lj], jz1);
        const C jx0 = jx[0][v], jx1 = jx[1][v];
        C rt[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            C rvol = -((dx[i] + dy[i]) + dz[i]);
            if (v == 1) rvol += A.forcing;
            if constexpr (sizeof(C) == 8) {
                if (A.flags & kRoundRhs) rvol = (C)(float)rvol;
            }
            // lifting -(j_L g_L' + j_R g_R') jac of the six faces (rk.cu:12-25)
            C r = fma(-jx0, A.sc.gl[0][i], rvol);
            r = fma(-jx1, A.sc.gr[0][i], r);
            r = fma(-jy0[i], A.sc.gl[1][lj], r);
            r = fma(-jy1[i], A.sc.gr[1][lj], r);
            r = fma(-jz0[i], A.sc.gl[2][lk], r);
            rt[i] = fma(-jz1[i], A.sc.gr[2][lk], r);
        }
        S* dst = A.u_out + v * m.npts + ec * NE + 4 * l;
        if (defer) {
            stg4<S, C>(dst, rt);
            continue;
        }
        P un[4], u0v[4], out[4];
        ldg4<S, P>(A.u_in + v * m.npts + ec * NE + 4 * l, un);
        if (A.flags & kHasU0) ldc4<S, P>(A.u0 + v * m.npts + ec * NE + 4 * l, u0v);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            P o = A.rb * un[i] + A.rc * (P)rt[i];
            if (A.flags & kHasU0) o = A.ra * u0v[i] + A.rb * un[i] + A.rc * (P)rt[i];
            out[i] = o;
        }
        stg4<S, P>(dst, out);
    }
}

// One tile of phase A: EPB elements starting at A.e0 + tile * EPB, LPE
// threads each. Called by every thread of the block (it synchronises).
template <class M, int FLUX, int EPB, bool FEAT = false, class PA>
__device__ __forceinline__ void stage_a_tile(const PA& A, unsigned char* smem_raw, long long tile) {
    using S = typename PA::S_t;
    using P = typename PA::P_t;
    using C = typename PA::C_t;
    const int l = threadIdx.x & (LPE - 1);
    const int es = threadIdx.x / LPE;
    const int swz = (es & 1) << 3;
    const LineIdx li = line_idx(l, swz);
    SlotA<P, C>& sm = reinterpret_cast<SlotA<P, C>*>(smem_raw)[es];
    const long long e = A.e0 + tile * EPB + es;
    const bool live = e < A.e1;
    const long long ec = live ? e : 0;
    const Mesh& m = A.m;
    int ex, ey, ez;
    elem_coords(m, ec, ex, ey, ez);
    const long long nxm = neighbour(m, ex, ey, ez, 0, 0), nxp = neighbour(m, ex, ey, ez, 0, 1);
    const long long nym = neighbour(m, ex, ey, ez, 1, 0), nyp = neighbour(m, ex, ey, ez, 1, 1);
    const long long nzm = neighbour(m, ex, ey, ez, 2, 0), nzp = neighbour(m, ex, ey, ez, 2, 1);

    // ---- P1: the element's x-lines -> smem (and kept for the x pass)
    P qx[NV][4];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        if (live) {
            ldg4<S, P>(A.u_in + v * m.npts + ec * NE + 4 * l, qx[v]);
        } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) qx[v][a] = (P)1.0;
        }
        st4s(&sm.u[v][sw(4 * l, swz)], qx[v]);
    }
    __syncthreads();
    if constexpr (FEAT) stage_a_features(A, sm, ec, l, swz, live, qx);

    // ---- P2-P4: face values, gradient, interface fluxes per direction
    P tr[3][2][NV];   // own face values of this thread's lines (kept only for f32 state arithmetic)
    C jx[2][NV];      // this x-line's x-face corrections
    C fi[3][NV];      // interface fluxes at the minus faces of this thread's lines
    line_pass<M, FLUX, 0>(A, sm, ec, l, li, live, nxm, nxp, tr[0][0], tr[0][1], jx, fi[0], qx);
    line_pass<M, FLUX, 1>(A, sm, ec, l, li, live, nym, nyp, tr[1][0], tr[1][1], jx, fi[1], qx);
    __syncthreads();   // the x and y gradients, read by the z faces
    line_pass<M, FLUX, 2>(A, sm, ec, l, li, live, nzm, nzp, tr[2][0], tr[2][1], jx, fi[2], qx);
    __syncthreads();

    // ---- P5: viscous face fluxes of the x and y faces, face records (the z
    // faces are done in the z pass)
    face_grad_pass<M, 0>(A, sm, ec, l, li, false, false, live, tr[0][0], tr[0][1], jx, fi[0]);
    face_grad_pass<M, 1>(A, sm, ec, l, li, nym < 0, nyp < 0, live, tr[1][0], tr[1][1], jx, fi[1]);
    __syncthreads();

    // ---- P6: pointwise fluxes of the x-line's points (own points only; the
    // point order is rotated by k so the 16 lanes of an element hit distinct
    // banks). F_y, F_z -> smem for the y / z divergences; the x-line's F_x
    // never leaves the thread: its x-divergence is accumulated here (point i
    // contributes column i of the x derivative) and kept until P8.
    C divx[NV][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int a = 0; a < 4; ++a) divx[v][a] = (C)0;
    {
        const int lk = l >> 2;
#pragma unroll 1
        for (int it = 0; it < 4; ++it) {
            const int i = (it + lk) & 3;
            const int p = sw(4 * l + i, swz);
            C g[15];
#pragma unroll
            for (int c = 0; c < 15; ++c) g[c] = sm.g[c][p];
            P qp[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) qp[v] = sm.u[v][p];
            C praw;
            FaceState<C> s = make_face_state<M, C, P>(qp, praw);
            C F[3][NV];
            const C mu = viscosity<M>(A.mu, A.suth, s);
            volume_fluxes<C>(s, praw, g, mu, heat_coeff<M>(mu, A.kappa), F);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                sm.g[v][p] = F[1][v];
                sm.g[5 + v][p] = F[2][v];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const C d = A.sc.d[0][a * 4 + i];
#pragma unroll
                for (int v = 0; v < NV; ++v) divx[v][a] = fma(d, F[0][v], divx[v][a]);
            }
        }
    }
    __syncthreads();

    // ---- P7 + P8: y / z divergences, RHS, lifting, RK combination (or the
    // RHS alone for phase B)
    if (live) stage_a_update(A, sm, ec, l, swz, divx, jx);
}

// Blocks per SM the register budget is set for. f32 state arithmetic and
// fluxes (the all-f32 pipeline, and the reference's default of an f64 state
// with f32 arithmetic): at most 128 registers per thread, so that 8 blocks of
// 4 elements (16 of 2) fit per SM, the occupancy the shared memory allows
// (u64/c32 at 64^3: phase A 1161 us at the 5 blocks its free choice of 198
// registers allowed, 931 us at 8; its SLAU2 fast-math kernel does not spill,
// some IEEE, AUSM+ and Sutherland variants spill 8-72 bytes). Mixed precision (f64 state, f32
// fluxes): 6 blocks of 4 elements, at most 168 registers (left free, the
// compiler takes 190 and 5 blocks fit: 10% slower at 96^3; 7 blocks spill and
// are 9% slower). Slots with f64 gradients are larger; shared memory bounds
// those kernels first.
template <class S, class P, class C, int EPB>
constexpr int stage_a_min_blocks() {
    if (sizeof(P) == 4 && sizeof(C) == 4) return 32 / EPB;
    if (sizeof(S) == 8 && sizeof(P) == 8 && sizeof(C) == 4) return 24 / EPB;
    return 1;
}

template <class S, class P, class C, class M, int FLUX, int EPB, bool FEAT = false>
__global__ void __launch_bounds__(LPE * EPB, (stage_a_min_blocks<S, P, C, EPB>())) stage_a_kernel(const StageAParams<S, P, C> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // the closure network launched next may start its prologue (and prefetch
    // its weights) on SMs this grid no longer needs; it reads the features
    // and the RHS only after griddepcontrol.wait, i.e. after this grid
    if constexpr (FEAT) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    stage_a_tile<M, FLUX, EPB, FEAT>(A, smem_raw, blockIdx.x);
}

template <class S, class P, class C>
struct StageBParams {
    using S_t = S;
    using P_t = P;
    using C_t = C;
    S* u_out;
    const S* rhs;   // deferred RK: phase A's RHS
    const S* u_in;
    const S* u0;
    const C* fv;
    const C* fi;
    Mesh m;
    Tab<C> tc;
    C jac[3];
    P ra, rb, rc;
    int flags;
    long long e0, e1;   // element range of this launch
};

// Phase B: the neighbour-dependent part of the face corrections,
//   plus faces:  j += F_I - 1/2 Fv_nbr (the plus neighbour's minus-face record)
//   minus faces: j += -1/2 Fv_nbr (the minus neighbour's plus-face record)
// lifted with -(j g') jac (rk.cu:12-25) over the element's non-wall faces and
// added to the new state (times rc), or (deferred RK) folded into
// u_out = ra*u0 + rb*u_in + rc*(RHS + lift). 16 threads per element, each the
// x-line l = j + 4k (128-bit accesses).
// Scalar load of data written earlier by the same kernel (COH) or by an
// earlier launch; phase B reads each face record and RHS value once, so the
// latter loads are evict-first (ld.global.cs): the L2 keeps the new state for
// the next phase A instead (48^3 f32: phase B 117.6 -> 117.0 us).
template <bool COH, class T>
__device__ __forceinline__ T ldf(const T* p) {
    if constexpr (COH)
        return *p;
    else
        return __ldcs(p);
}

// 4-wide load of data read once (evict-first: the face records and the RHS
// phase B consumes), or coherent inside a persistent kernel (COH)
template <bool COH, class S, class P>
__device__ __forceinline__ void ld4once(const S* p, P* q) {
    if constexpr (COH || sizeof(S) != 4) {
        ldc4<S, P>(p, q);
    } else {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
        q[0] = (P)v.x; q[1] = (P)v.y; q[2] = (P)v.z; q[3] = (P)v.w;
    }
}

// One tile of phase B: EPB elements starting at B.e0 + tile * EPB. COH: the
// face buffers and the RHS were written by this same launch (a persistent
// kernel after its grid barrier), so they are read through the coherent path.
// Per-element context of phase B: the element, its x-line and its neighbours.
template <class C>
struct BCtx {
    long long e, nxm, nxp, nym, nyp, nzm, nzp;
    int l, lj, lk;
    C hx, hy, hz;
};

template <class PB, class C = typename PB::C_t>
__device__ __forceinline__ BCtx<C> b_ctx(const PB& B, long long e, int l) {
    BCtx<C> x;
    const Mesh& m = B.m;
    int ex, ey, ez;
    elem_coords(m, e, ex, ey, ez);
    x.e = e;
    x.l = l;
    x.lj = l & 3;
    x.lk = l >> 2;
    x.nxm = neighbour(m, ex, ey, ez, 0, 0);
    x.nxp = neighbour(m, ex, ey, ez, 0, 1);
    x.nym = neighbour(m, ex, ey, ez, 1, 0);
    x.nyp = neighbour(m, ex, ey, ez, 1, 1);
    x.nzm = neighbour(m, ex, ey, ez, 2, 0);
    x.nzp = neighbour(m, ex, ey, ez, 2, 1);
    x.hx = (C)0.5 * B.jac[0];
    x.hy = (C)0.5 * B.jac[1];
    x.hz = (C)0.5 * B.jac[2];
    return x;
}

// Phase B of variable v on the x-line x.l of element x.e, in two halves:
// b_load gathers everything the update reads (the lifted neighbour terms
// accumulated from the face records, and the RHS / state values), b_store
// forms the new state and stores it. A thread that handles several variables
// issues all their loads before its first store.
template <class P, class C>
struct BVar {
    C acc[4];   // lifted neighbour face terms
    C r[4];     // deferred RK: phase A's RHS
    P un[4];    // deferred RK: u_in; otherwise the current u_out
    P u0[4];
};

template <bool COH, class PB, class C = typename PB::C_t, class P = typename PB::P_t>
__device__ __forceinline__ BVar<P, C> b_load(const PB& B, const BCtx<C>& x, int v) {
    using S = typename PB::S_t;
    const Mesh& m = B.m;
    const bool defer = (B.flags & kDeferRK) != 0;
    const long long e = x.e, nxm = x.nxm, nxp = x.nxp, nym = x.nym, nyp = x.nyp, nzm = x.nzm, nzp = x.nzp;
    const int l = x.l, lj = x.lj, lk = x.lk;
    const C hx = x.hx, hy = x.hy, hz = x.hz;
    BVar<P, C> d;
#pragma unroll
    for (int i = 0; i < 4; ++i) d.acc[i] = (C)0;
    // plus faces: the plus neighbours' minus-face records F_I - 1/2 Fv
    {
        const C f0 = ldf<COH>(B.fi + ((nxp * 3 + 0) * NV + v) * NF + l);
#pragma unroll
        for (int i = 0; i < 4; ++i) d.acc[i] = fma(-B.jac[0] * B.tc.gR[i], f0, d.acc[i]);
    }
    if (nyp >= 0) {
        C w[4];
        ld4once<COH, C, C>(B.fi + ((nyp * 3 + 1) * NV + v) * NF + 4 * lk, w);
        const C c = -B.jac[1] * B.tc.gR[lj];
#pragma unroll
        for (int i = 0; i < 4; ++i) d.acc[i] = fma(c, w[i], d.acc[i]);
    }
    {
        C w[4];
        ld4once<COH, C, C>(B.fi + ((nzp * 3 + 2) * NV + v) * NF + 4 * lj, w);
        const C c = -B.jac[2] * B.tc.gR[lk];
#pragma unroll
        for (int i = 0; i < 4; ++i) d.acc[i] = fma(c, w[i], d.acc[i]);
    }
    if (v > 0) {
        // minus faces: the minus neighbours' viscous fluxes at their plus faces
        const int q = v - 1;
        {
            const C a0 = ldf<COH>(B.fv + ((nxm * 3 + 0) * 4 + q) * NF + l);
#pragma unroll
            for (int i = 0; i < 4; ++i) d.acc[i] = fma(hx * B.tc.gL[i], a0, d.acc[i]);
        }
        if (nym >= 0) {
            C w[4];
            ld4once<COH, C, C>(B.fv + ((nym * 3 + 1) * 4 + q) * NF + 4 * lk, w);
            const C c = hy * B.tc.gL[lj];
#pragma unroll
            for (int i = 0; i < 4; ++i) d.acc[i] = fma(c, w[i], d.acc[i]);
        }
        {
            C w[4];
            ld4once<COH, C, C>(B.fv + ((nzm * 3 + 2) * 4 + q) * NF + 4 * lj, w);
            const C c = hz * B.tc.gL[lk];
#pragma unroll
            for (int i = 0; i < 4; ++i) d.acc[i] = fma(c, w[i], d.acc[i]);
        }
    }
    const long long off = v * m.npts + e * NE + 4 * l;
    if (defer) {
        ld4once<COH, S, C>(B.rhs + off, d.r);
        ldg4<S, P>(B.u_in + off, d.un);
        if (B.flags & kHasU0) ldc4<S, P>(B.u0 + off, d.u0);
    } else {
        ldc4<S, P>(B.u_out + off, d.un);
    }
    return d;
}

template <class PB, class C = typename PB::C_t, class P = typename PB::P_t>
__device__ __forceinline__ void b_store(const PB& B, const BCtx<C>& x, int v, const BVar<P, C>& d) {
    using S = typename PB::S_t;
    const bool defer = (B.flags & kDeferRK) != 0;
    const long long off = v * B.m.npts + x.e * NE + 4 * x.l;
    P out[4];
    if (defer) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const C rt = d.r[i] + d.acc[i];
            P o = B.rb * d.un[i] + B.rc * (P)rt;
            if (B.flags & kHasU0) o = B.ra * d.u0[i] + B.rb * d.un[i] + B.rc * (P)rt;
            out[i] = o;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] = d.un[i] + B.rc * (P)d.acc[i];
    }
    stg4<S, P>(B.u_out + off, out);
}

template <bool COH, class PB, class C = typename PB::C_t>
__device__ __forceinline__ void stage_b_var(const PB& B, const BCtx<C>& x, int v) {
    b_store(B, x, v, b_load<COH>(B, x, v));
}

// One tile of phase B: EPB elements starting at B.e0 + tile * EPB, 16
// threads (x-lines) each, all five variables per thread. COH: the face
// buffers and the RHS were written by this same launch (a persistent kernel
// after its grid barrier), so they are read through the coherent path.
template <int EPB, bool COH, class PB>
__device__ __forceinline__ void stage_b_tile(const PB& B, long long tile) {
    const int l = threadIdx.x & (LPE - 1);
    const long long e = B.e0 + tile * EPB + threadIdx.x / LPE;
    if (e >= B.e1) return;
    const auto x = b_ctx(B, e, l);
    if constexpr (COH) {
        // inside the persistent ensemble kernel (phase A's occupancy): all
        // five variables' loads first for memory-level parallelism, then the
        // stores (6.89 -> 6.05 ms per step on the 64-box ensemble)
        using P = typename PB::P_t;
        using C = typename PB::C_t;
        BVar<P, C> d[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v] = b_load<COH>(B, x, v);
#pragma unroll
        for (int v = 0; v < NV; ++v) b_store(B, x, v, d[v]);
    } else {
        // a launch of its own: one variable at a time keeps the registers,
        // and with them the occupancy, low
#pragma unroll
        for (int v = 0; v < NV; ++v) stage_b_var<COH>(B, x, v);
    }
}

template <class S, class P, class C, int EPB>
__global__ void __launch_bounds__(LPE * EPB) stage_b_kernel(const StageBParams<S, P, C> B) {
    stage_b_tile<EPB, false>(B, blockIdx.x);
}

// Phase B with one thread per (element, variable, x-line): 80 threads per
// element; a warp holds two elements' lines of one variable. Blocks walk
// the elements in reverse order: phase A's last RHS and face records (the
// highest elements) are still in L2 when phase B starts, and phase B's last
// stores (the lowest elements) are what the next phase A reads first
// (48^3 f32: phase B 120.9 -> 117.5 us, phase A 263.0 -> 262.4 us).
template <class S, class P, class C, int EPB>
__global__ void __launch_bounds__(LPE * NV * EPB) stage_b_split_kernel(const StageBParams<S, P, C> B) {
    const int g = threadIdx.x / LPE;
    const int v = g / EPB;
    const long long e = B.e0 + (long long)(gridDim.x - 1 - blockIdx.x) * EPB + (g - v * EPB);
    if (e >= B.e1) return;
    stage_b_var<false>(B, b_ctx(B, e, threadIdx.x & (LPE - 1)), v);
}

}  // namespace od
