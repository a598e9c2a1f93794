// FR P=3 stage kernels for sm_100a.
//
// One SSP-RK3 stage of the reference (src/solver.rs:262-317) is the
// volume kernel, three face kernels (+ the y-wall kernel) and the RK kernel
// (src/cuda/rhs.cu:344-739, src/cuda/rk.cu:85-115): seven passes over HBM
// with 6 gradient slice arrays and 6 face-correction arrays in between.
// Here a stage is two element-local phases:
//
//  phase A (one element per 64 threads)
//    - stage the element's 5x64 state in shared memory,
//    - face values of the element and of its six neighbours (BR1 common
//      solution, slip-wall mirror of rhs.cu:111-114),
//    - corrected gradient (rhs.cu:373-455) kept in registers + shared memory,
//    - volume divergence of F_euler - F_viscous (rhs.cu:229-266),
//    - at all 6 faces: the interface flux F_I from the two face states, the
//      element's own Euler and viscous face fluxes; the element's face
//      correction j = F_I - 1/2 (Fv_own + Fv_nbr) - (Fe_own - Fv_own)
//      (rhs.cu:273-297) is formed up to its -1/2 Fv_nbr term,
//    - correction lifting with the Radau g' (rk.cu:12-25) and the RK
//      combination a*u0 + b*u + c*(RHS + lift) (rk.cu:27-83),
//    - the element's own viscous face flux (4 non-zero components) is
//      written to a small face buffer for its neighbours;
//  phase B (one element per 64 threads)
//    - adds c * lift(-1/2 Fv_nbr) for the element's non-wall faces.
//
// Only the viscous flux needs the neighbour's *gradient*, which depends on
// the neighbour's neighbours; splitting it out is what lets everything else
// run in one pass. Phase B is skipped when mu == 0.
//
// Types: S = stored state, P = state arithmetic (face values, pressure
// recovery, RK accumulation), C = flux arithmetic. Reference-compatible
// pipelines use P == C; the mixed-precision form uses S = P = double with
// C = float.
#pragma once

#include "od_launch.h"
#include "od_physics.cuh"

namespace od {

constexpr int NP = 4;   // points per direction
constexpr int NF = 16;  // points per face
constexpr int NE = 64;  // points per element
constexpr int NV = 5;   // conserved variables

template <class T>
struct Tab {
    T D[16];   // D[a*4+m] = l'_m(x_a)
    T eL[4];   // l_m(-1)
    T eR[4];   // l_m(+1)
    T gL[4];   // Radau g_L'(x_a)
    T gR[4];   // Radau g_R'(x_a)
};

struct Mesh {
    int nx, ny, nz, y_wall;
    long long nelem, npts;
};

// point index inside an element: i + 4 j + 16 k
__device__ __forceinline__ int pid(int i, int j, int k) { return i + NP * j + NF * k; }

// point m of the direction-d line through face point fp
// (fp = j + 4k for x, i + 4k for y, i + 4j for z, as the reference's faces)
__device__ __forceinline__ int line_pt(int d, int fp, int m) {
    const int a = fp & 3, b = fp >> 2;
    return d == 0 ? pid(m, a, b) : (d == 1 ? pid(a, m, b) : pid(a, b, m));
}

// Face value from the four samples of a line; one fixed FMA chain so that the
// two elements sharing a face compute bit-identical face states.
template <class T>
__device__ __forceinline__ T trace4(T q0, T q1, T q2, T q3, const T* c) {
    return fma(q3, c[3], fma(q2, c[2], fma(q1, c[1], q0 * c[0])));
}

// neighbour across face (d, side) or -1 for a slip wall
__device__ __forceinline__ long long neighbour(const Mesh& m, int ex, int ey, int ez, int d, int side) {
    int c[3] = {ex, ey, ez};
    const int n[3] = {m.nx, m.ny, m.nz};
    int tgt = c[d] + (side ? 1 : -1);
    if (d == 1 && m.y_wall && (tgt < 0 || tgt >= n[1])) return -1;
    if (tgt < 0) tgt += n[d];
    if (tgt >= n[d]) tgt -= n[d];
    c[d] = tgt;
    return (long long)c[0] + (long long)m.nx * ((long long)c[1] + (long long)m.ny * c[2]);
}

// Load the 4 samples of a neighbour's line from global memory.
template <class S, class P>
__device__ __forceinline__ void load_line(const S* __restrict__ base, int d, int fp, P* q) {
    if (d == 0) {
        const S* p = base + 4 * fp;
        if constexpr (sizeof(S) == 4) {
            float4 v = __ldg(reinterpret_cast<const float4*>(p));
            q[0] = (P)v.x; q[1] = (P)v.y; q[2] = (P)v.z; q[3] = (P)v.w;
        } else {
            double2 a = __ldg(reinterpret_cast<const double2*>(p));
            double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
            q[0] = (P)a.x; q[1] = (P)a.y; q[2] = (P)b.x; q[3] = (P)b.y;
        }
    } else {
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) q[mm] = (P)__ldg(base + line_pt(d, fp, mm));
    }
}

// which gradient components the direction-d viscous flux reads
__device__ __forceinline__ bool grad_used(int d, int c) {
    // x omits 8,10,13,14; y omits 5,9,12,14; z omits 4,6,12,13 (rhs.cu:129,151,169)
    const unsigned omit = d == 0 ? ((1u << 8) | (1u << 10) | (1u << 13) | (1u << 14))
                        : d == 1 ? ((1u << 5) | (1u << 9) | (1u << 12) | (1u << 14))
                                 : ((1u << 4) | (1u << 6) | (1u << 12) | (1u << 13));
    return !((omit >> c) & 1u);
}

// Shared-memory slot of one element in phase A.
template <class P, class C>
struct SlotA {
    P u[NV][NE];            // element state
    P tr[3][2][NV][NF];     // own face values  [dir][side][var][face pt]
    P nb[3][2][NV][NF];     // neighbour face values
    C g[15][NE];            // corrected gradient; reused for the volume fluxes F[3][5][64]
    C j[3][2][NV][NF];      // face corrections without the -1/2 Fv_nbr part
};

template <class S, class P, class C>
struct StageAParams {
    const S* u_in;
    const S* u0;
    S* u_out;
    C* fv;          // [elem][face 6][var 4][face pt 16]: own viscous face flux, components 1..4
    Mesh m;
    Tab<P> tp;
    Tab<C> tc;
    C jac[3];
    P ra, rb, rc;
    C mu, forcing;
    int flags;
};

// One face point of phase A, direction D.
template <int FLUX, int D, class S, class P, class C>
__device__ __forceinline__ void face_point(const StageAParams<S, P, C>& A, SlotA<P, C>& sm, long long e, int side,
                                           int fp, bool wall) {
    P qo[NV], qn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        qo[v] = sm.tr[D][side][v][fp];
        qn[v] = sm.nb[D][side][v][fp];
    }
    // own gradient at the face (the 11 components the D-flux reads)
    C gt[15];
    const C* ec = side ? A.tc.eR : A.tc.eL;
#pragma unroll
    for (int c = 0; c < 15; ++c) {
        if (!grad_used(D, c)) {
            gt[c] = (C)0;
            continue;
        }
        gt[c] = trace4(sm.g[c][line_pt(D, fp, 0)], sm.g[c][line_pt(D, fp, 1)], sm.g[c][line_pt(D, fp, 2)],
                       sm.g[c][line_pt(D, fp, 3)], ec);
    }
    FaceState<C> so = make_face_state<C, P>(qo);
    C praw_o = (C)raw_pressure<P>(qo[0], qo[1], qo[2], qo[3], qo[4]);
    C fvo[NV], feo[NV], jv[NV];
    viscous_flux<D>(so, praw_o, gt, A.mu, fvo);
    euler_flux<D>(so, feo);
    if (wall) {
        // slip wall: F = [0, 0, p_wall, 0, 0] with p_wall from the own flux
        // (rhs.cu:311-339); the viscous traction cancels exactly.
        C fw2 = feo[2] - so.q[2] * so.q[2] * so.ir;
#pragma unroll
        for (int v = 0; v < NV; ++v) jv[v] = -feo[v];
        jv[2] = fw2 - feo[2];
    } else {
        FaceState<C> sn = make_face_state<C, P>(qn);
        C fi[NV];
        if (side)
            interface_flux<FLUX, D>(so, sn, fi);
        else
            interface_flux<FLUX, D>(sn, so, fi);
#pragma unroll
        for (int v = 0; v < NV; ++v) jv[v] = fi[v] - feo[v] + (C)0.5 * fvo[v];
        C* out = A.fv + ((e * 6 + 2 * D + side) * 4) * NF + fp;
#pragma unroll
        for (int v = 1; v < NV; ++v) out[(v - 1) * NF] = fvo[v];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) sm.j[D][side][v][fp] = jv[v];
}

template <class S, class P, class C, int FLUX, int EPB>
__global__ void __launch_bounds__(64 * EPB) stage_a_kernel(const StageAParams<S, P, C> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int t = threadIdx.x & 63;
    const int es = threadIdx.x >> 6;
    SlotA<P, C>& sm = reinterpret_cast<SlotA<P, C>*>(smem_raw)[es];
    const long long e = (long long)blockIdx.x * EPB + es;
    const bool live = e < A.m.nelem;
    const long long ec = live ? e : 0;
    const Mesh& m = A.m;
    const int ex = (int)(ec % m.nx);
    const int ey = (int)((ec / m.nx) % m.ny);
    const int ez = (int)(ec / ((long long)m.nx * m.ny));
    const int ia[3] = {t & 3, (t >> 2) & 3, t >> 4};               // position along x, y, z
    const int fpa[3] = {ia[1] + 4 * ia[2], ia[0] + 4 * ia[2], ia[0] + 4 * ia[1]};  // face point per dir

    // ---- 1. state of this element
    P uin[NV];
    if (live) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            uin[v] = (P)A.u_in[v * m.npts + ec * NE + t];
            sm.u[v][t] = uin[v];
        }
    }
    long long nbr[3][2];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int s = 0; s < 2; ++s) nbr[d][s] = neighbour(m, ex, ey, ez, d, s);
    __syncthreads();

    // ---- 2. own and neighbour face values (3 dirs x 5 vars x 16 face pts)
    if (live) {
        for (int it = t; it < 240; it += 64) {
            const int d = it / 80;
            const int rem = it - d * 80;
            const int v = rem >> 4, fp = rem & 15;
            const P q0 = sm.u[v][line_pt(d, fp, 0)], q1 = sm.u[v][line_pt(d, fp, 1)];
            const P q2 = sm.u[v][line_pt(d, fp, 2)], q3 = sm.u[v][line_pt(d, fp, 3)];
            const P oL = trace4(q0, q1, q2, q3, A.tp.eL);
            const P oR = trace4(q0, q1, q2, q3, A.tp.eR);
            P nL, nR;
            const P refl = (v > 0 && v < 4) ? (P)-1.0 : (P)1.0;
            if (nbr[d][0] >= 0) {
                P q[4];
                load_line<S, P>(A.u_in + v * m.npts + nbr[d][0] * NE, d, fp, q);
                nL = trace4(q[0], q[1], q[2], q[3], A.tp.eR);
            } else {
                nL = oL * refl;
            }
            if (nbr[d][1] >= 0) {
                P q[4];
                load_line<S, P>(A.u_in + v * m.npts + nbr[d][1] * NE, d, fp, q);
                nR = trace4(q[0], q[1], q[2], q[3], A.tp.eL);
            } else {
                nR = oR * refl;
            }
            sm.tr[d][0][v][fp] = oL;
            sm.tr[d][1][v][fp] = oR;
            sm.nb[d][0][v][fp] = nL;
            sm.nb[d][1][v][fp] = nR;
        }
    }
    __syncthreads();

    // ---- 3. corrected gradient at this point (BR1, rhs.cu:373-461)
    C Dr[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int mm = 0; mm < 4; ++mm) Dr[d][mm] = A.tc.D[ia[d] * 4 + mm];
    C gl[3], gr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        gl[d] = A.tc.gL[ia[d]];
        gr[d] = A.tc.gR[ia[d]];
    }
    C g[15];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int fp = fpa[d];
            C der = (C)0;
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) der = fma(Dr[d][mm], (C)sm.u[v][line_pt(d, fp, mm)], der);
            const P tl = sm.tr[d][0][v][fp], tr = sm.tr[d][1][v][fp];
            const C jl = (C)((P)0.5 * (sm.nb[d][0][v][fp] + tl) - tl);
            const C jr = (C)((P)0.5 * (sm.nb[d][1][v][fp] + tr) - tr);
            C gv = der * A.jac[d];
            gv += jl * gl[d] * A.jac[d];
            gv += jr * gr[d] * A.jac[d];
            if constexpr (sizeof(C) == 8) {
                if (A.flags & kRoundQ) gv = (C)(float)gv;
            }
            g[3 * v + d] = gv;
            sm.g[3 * v + d][t] = gv;
        }
    }
    __syncthreads();

    // ---- 4. face points: interface flux, own fluxes, corrections
    if (live) {
        for (int it = t; it < 96; it += 64) {
            const int d = it >> 5, side = (it >> 4) & 1, fp = it & 15;
            const bool wall = d == 1 && nbr[1][side] < 0;
            if (d == 0)
                face_point<FLUX, 0>(A, sm, ec, side, fp, wall);
            else if (d == 1)
                face_point<FLUX, 1>(A, sm, ec, side, fp, wall);
            else
                face_point<FLUX, 2>(A, sm, ec, side, fp, wall);
        }
    }
    // ---- 5. volume fluxes at this point
    C F[3][NV];
    {
        P qp[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) qp[v] = sm.u[v][t];
        FaceState<C> s = make_face_state<C, P>(qp);
        C praw = (C)raw_pressure<P>(qp[0], qp[1], qp[2], qp[3], qp[4]);
        volume_fluxes<C>(s, praw, g, A.mu, F);
    }
    __syncthreads();  // face points are done reading the gradient
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.g[d * NV + v][t] = F[d][v];
    __syncthreads();

    // ---- 6. divergence, lifting and the RK combination
    if (!live) return;
    P u0v[NV];
    if (A.flags & kHasU0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) u0v[v] = (P)A.u0[v * m.npts + ec * NE + t];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        C div = (C)0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int fp = fpa[d];
            const C* Fr = sm.g[d * NV + v];
            C df = (C)0;
#pragma unroll
            for (int mm = 0; mm < 4; ++mm) df = fma(Dr[d][mm], Fr[line_pt(d, fp, mm)], df);
            div += df * A.jac[d];
        }
        C rvol = -div;
        if (v == 1) rvol += A.forcing;
        if constexpr (sizeof(C) == 8) {
            if (A.flags & kRoundRhs) rvol = (C)(float)rvol;
        }
        C corr[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int fp = fpa[d];
            corr[d] = -(sm.j[d][0][v][fp] * gl[d] * A.jac[d]) - (sm.j[d][1][v][fp] * gr[d] * A.jac[d]);
        }
        const C rtot = rvol + (corr[0] + corr[1] + corr[2]);
        P out = A.rb * uin[v] + A.rc * (P)rtot;
        if (A.flags & kHasU0) out = A.ra * u0v[v] + A.rb * uin[v] + A.rc * (P)rtot;
        A.u_out[v * m.npts + ec * NE + t] = (S)out;
    }
}

template <class S, class P, class C>
struct StageBParams {
    S* u_out;
    const C* fv;
    Mesh m;
    Tab<C> tc;
    C jac[3];
    P rc;
};

// Phase B: u_out += rc * lift(-1/2 Fv_nbr) over the element's non-wall faces.
template <class S, class P, class C, int EPB>
__global__ void __launch_bounds__(64 * EPB) stage_b_kernel(const StageBParams<S, P, C> B) {
    const int t = threadIdx.x & 63;
    const long long e = (long long)blockIdx.x * EPB + (threadIdx.x >> 6);
    const Mesh& m = B.m;
    if (e >= m.nelem) return;
    const int ex = (int)(e % m.nx);
    const int ey = (int)((e / m.nx) % m.ny);
    const int ez = (int)(e / ((long long)m.nx * m.ny));
    const int ia[3] = {t & 3, (t >> 2) & 3, t >> 4};
    const int fpa[3] = {ia[1] + 4 * ia[2], ia[0] + 4 * ia[2], ia[0] + 4 * ia[1]};
    C acc[4] = {(C)0, (C)0, (C)0, (C)0};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const long long nb = neighbour(m, ex, ey, ez, d, side);
            if (nb < 0) continue;
            const C w = (C)0.5 * B.jac[d] * (side ? B.tc.gR[ia[d]] : B.tc.gL[ia[d]]);
            // the neighbour's record of the shared face is its opposite side
            const C* src = B.fv + ((nb * 6 + 2 * d + (1 - side)) * 4) * NF + fpa[d];
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[v] = fma(w, __ldg(src + v * NF), acc[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        S* p = B.u_out + (v + 1) * m.npts + e * NE + t;
        *p = (S)((P)*p + B.rc * (P)acc[v]);
    }
}

}  // namespace od
