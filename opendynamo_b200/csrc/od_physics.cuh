// Pointwise compressible Navier-Stokes physics for the FR P=3 step path.
//
// Same mathematics as the reference's device library
// (src/cuda/device_functions.cuh): ideal gas gamma = 1.4, Pr = 0.72,
// Stokes hypothesis, heat flux -mu*gamma/(Pr*(gamma-1)) * grad(p/rho),
// pressure clamped at 1e-7 in the inviscid fluxes and sound speeds, and the
// Rusanov / AUSM+ / SLAU2 interface fluxes on axis-aligned normals.
//
// Laid out for the GPU rather than per call: the primitive variables of a
// point (1/rho, velocity, pressure) are formed once and shared by the Euler
// flux, the viscous flux of all three directions and the Riemann solvers.
// Normals are axis-aligned, so the direction is a template argument and the
// normal velocity is a register pick, not a dot product.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace od {

enum Flux : int { kSlau2 = 0, kAusmPlus = 1, kRusanov = 2 };

// Division / reciprocal / square root policy. MathIeee: correctly rounded
// (the reference with fast_math = false, and every f64 operation).
// MathFast: for f32 operands the approximate PTX forms (rcp.approx,
// sqrt.approx, ~1-2 ulp), the arithmetic of the reference's default
// --use_fast_math build; f64 operands stay IEEE (fast math does not touch them).
struct MathIeee {
    static constexpr bool kSutherland = false;
    template <class T>
    static __device__ __forceinline__ T rcp(T x) { return (T)1.0 / x; }
    template <class T>
    static __device__ __forceinline__ T div(T a, T b) { return a / b; }
    template <class T>
    static __device__ __forceinline__ T sqrt(T x) { return ::sqrt(x); }
};

struct MathFast {
    static constexpr bool kSutherland = false;
    template <class T>
    static __device__ __forceinline__ T rcp(T x) {
        if constexpr (sizeof(T) == 4) {
            float r;
            asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
            return r;
        } else {
            return (T)1.0 / x;
        }
    }
    template <class T>
    static __device__ __forceinline__ T div(T a, T b) {
        if constexpr (sizeof(T) == 4) return a * rcp(b);
        else return a / b;
    }
    template <class T>
    static __device__ __forceinline__ T sqrt(T x) {
        if constexpr (sizeof(T) == 4) {
            float r;
            asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
            return r;
        } else {
            return ::sqrt(x);
        }
    }
};

// A math policy with Sutherland's law switched on (a separate kernel variant,
// so the constant-viscosity kernels carry no trace of it).
template <class Base>
struct WithSutherland : Base {
    static constexpr bool kSutherland = true;
};

template <class C>
struct Gas {
    static __device__ __forceinline__ C gamma() { return (C)1.4; }
    static __device__ __forceinline__ C gm1() { return (C)1.4 - (C)1.0; }
    static __device__ __forceinline__ C pr() { return (C)0.72; }
};

template <class C>
__device__ __forceinline__ C cmax(C a, C b) { return a > b ? a : b; }
template <class C>
__device__ __forceinline__ C cmin(C a, C b) { return a < b ? a : b; }

// Raw pressure (gamma-1)(E - |m|^2 / (2 rho)); the viscous flux uses it unclamped.
template <class M, class P>
__device__ __forceinline__ P raw_pressure(P r, P m0, P m1, P m2, P E) {
    P ke = M::div((P)0.5 * (m0 * m0 + m1 * m1 + m2 * m2), r);
    return Gas<P>::gm1() * (E - ke);
}

template <class C>
__device__ __forceinline__ C clamp_p(C p) { return cmax((C)1e-7, p); }

// Face state in compute type: conserved variables, 1/rho, velocity and the
// clamped pressure (recovered in the state precision P by the caller).
template <class C>
struct FaceState {
    C q[5];
    C ir;
    C vel[3];
    C p;   // clamped
};

template <class M, class C, class P>
__device__ __forceinline__ FaceState<C> make_face_state(const P* qp, C& praw_out) {
    FaceState<C> s;
#pragma unroll
    for (int v = 0; v < 5; ++v) s.q[v] = (C)qp[v];
    P praw = raw_pressure<M, P>(qp[0], qp[1], qp[2], qp[3], qp[4]);
    praw_out = (C)praw;
    s.p = clamp_p<C>((C)praw);
    s.ir = M::rcp(s.q[0]);
    s.vel[0] = s.q[1] * s.ir;
    s.vel[1] = s.q[2] * s.ir;
    s.vel[2] = s.q[3] * s.ir;
    return s;
}

// Inviscid flux along axis D.
template <int D, class C>
__device__ __forceinline__ void euler_flux(const FaceState<C>& s, C* f) {
    C vn = s.vel[D];
    f[0] = s.q[1 + D];
    f[1] = s.q[1] * vn;
    f[2] = s.q[2] * vn;
    f[3] = s.q[3] * vn;
    f[1 + D] += s.p;
    f[4] = vn * (s.q[4] + s.p);
}

// Inviscid flux along axis d (d known after unrolling).
template <class C>
__device__ __forceinline__ void euler_flux_dyn(const FaceState<C>& s, int d, C* f) {
    C vn = s.vel[d];
    f[0] = s.q[1 + d];
    f[1] = s.q[1] * vn;
    f[2] = s.q[2] * vn;
    f[3] = s.q[3] * vn;
    f[1 + d] += s.p;
    f[4] = vn * (s.q[4] + s.p);
}

template <class M, class C>
__device__ __forceinline__ C sound_speed(C p, C r) {
    return M::sqrt(cmax((C)0.0, M::div(Gas<C>::gamma() * p, cmax((C)1e-7, r))));
}

// Dynamic viscosity at a point. Policies without kSutherland: constant mu
// (the reference's MU_REF, src/cuda/constants.cuh:42). Otherwise Sutherland's law
//   mu = mu_ref * T^(3/2) * (1 + S) / (T + S),
// T = gamma * p / rho the temperature in units of the reference temperature
// (rho = 1, c = 1 there) and S = s_suth / t_ref (config.toml [physics]).
// An extension: the reference parses viscosity_model but no kernel reads it.
template <class M, class C>
__device__ __forceinline__ C viscosity(C mu, C suth, const FaceState<C>& s) {
    if constexpr (!M::kSutherland) {
        return mu;
    } else {
        const C T = Gas<C>::gamma() * s.p * s.ir;
        return mu * T * M::sqrt(T) * M::div((C)1.0 + suth, T + suth);
    }
}

// Heat-flux coefficient mu gamma / (Pr (gamma - 1)), in the reference's
// operation order (device_functions.cuh:44). Constant viscosity: the value
// formed once per launch on the host with the same IEEE operations
// (kappa_const, heat_coeff_host); Sutherland's law: per point.
template <class M, class C>
__device__ __forceinline__ C heat_coeff(C mu, C kappa_const) {
    if constexpr (!M::kSutherland)
        return kappa_const;
    else
        return mu * Gas<C>::gamma() / (Gas<C>::pr() * Gas<C>::gm1());
}

template <class C>
__host__ inline C heat_coeff_host(C mu) {
    return mu * (C)1.4 / ((C)0.72 * ((C)1.4 - (C)1.0));
}

// Viscous flux along axis D at a face point from the state and the
// 15-component conserved gradient g[3*var + axis] (only the 11 components
// the D-flux reads are touched); kappa = heat_coeff(mu).
template <int D, class C>
__device__ __forceinline__ void viscous_flux(const FaceState<C>& s, C praw, const C* g, C mu, C kappa, C* f) {
    const C ir = s.ir;
    // d(vel_a)/d(x_b) for the pairs the D-flux needs
    auto dv = [&](int a, int b) -> C { return (g[3 * (1 + a) + b] - s.vel[a] * g[b]) * ir; };
    C div = dv(0, 0) + dv(1, 1) + dv(2, 2);
    C tau[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a == D)
            tau[a] = mu * ((C)2.0 * dv(D, D) - (C)2.0 / (C)3.0 * div);
        else
            tau[a] = mu * (dv(a, D) + dv(D, a));
    }
    C ke = (C)0.5 * (s.q[1] * s.vel[0] + s.q[2] * s.vel[1] + s.q[3] * s.vel[2]);
    C dke = (s.q[1] * g[3 + D] + s.q[2] * g[6 + D] + s.q[3] * g[9 + D]) * ir - ke * g[D] * ir;
    C dp = Gas<C>::gm1() * (g[12 + D] - dke);
    C heat = -kappa * (dp * ir - praw * g[D] * ir * ir);
    f[0] = (C)0.0;
    f[1] = tau[0];
    f[2] = tau[1];
    f[3] = tau[2];
    f[4] = s.vel[0] * tau[0] + s.vel[1] * tau[1] + s.vel[2] * tau[2] - heat;
}

// Volume fluxes of all three directions at a solution point:
// out[d][v] = F_euler,d - F_viscous,d. The velocity gradient, stress tensor
// and heat flux are formed once and shared by the three directions.
template <class C>
__device__ __forceinline__ void volume_fluxes(const FaceState<C>& s, C praw, const C* g, C mu, C kappa,
                                              C out[3][5]) {
    const C ir = s.ir;
    C dvel[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) dvel[a][b] = (g[3 * (1 + a) + b] - s.vel[a] * g[b]) * ir;
    C div = dvel[0][0] + dvel[1][1] + dvel[2][2];
    C tau[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        tau[a][a] = mu * ((C)2.0 * dvel[a][a] - (C)2.0 / (C)3.0 * div);
#pragma unroll
        for (int b = a + 1; b < 3; ++b) {
            C t = mu * (dvel[a][b] + dvel[b][a]);
            tau[a][b] = t;
            tau[b][a] = t;
        }
    }
    C ke = (C)0.5 * (s.q[1] * s.vel[0] + s.q[2] * s.vel[1] + s.q[3] * s.vel[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        C vn = s.vel[d];
        C dke = (s.q[1] * g[3 + d] + s.q[2] * g[6 + d] + s.q[3] * g[9 + d]) * ir - ke * g[d] * ir;
        C dp = Gas<C>::gm1() * (g[12 + d] - dke);
        C heat = -kappa * (dp * ir - praw * g[d] * ir * ir);
        // (F_euler) - (F_viscous), each formed first as the reference does
        C fe[5];
        euler_flux_dyn(s, d, fe);
        out[d][0] = fe[0];
        out[d][1] = fe[1] - tau[0][d];
        out[d][2] = fe[2] - tau[1][d];
        out[d][3] = fe[3] - tau[2][d];
        out[d][4] = fe[4] - (s.vel[0] * tau[0][d] + s.vel[1] * tau[1][d] + s.vel[2] * tau[2][d] - heat);
    }
}

// ---- interface fluxes (axis-aligned normal D, left state L, right state R) ----

template <class M, int D, class C>
__device__ __forceinline__ void rusanov(const FaceState<C>& L, const FaceState<C>& R, C* f) {
    C vnL = L.vel[D], vnR = R.vel[D];
    C smax = cmax(fabs(vnL) + sound_speed<M>(L.p, L.q[0]), fabs(vnR) + sound_speed<M>(R.p, R.q[0]));
    C fL[5], fR[5];
    euler_flux<D>(L, fL);
    euler_flux<D>(R, fR);
#pragma unroll
    for (int v = 0; v < 5; ++v) f[v] = (C)0.5 * (fL[v] + fR[v] - smax * (R.q[v] - L.q[v]));
}

template <class M, int D, class C>
__device__ __forceinline__ void ausm_plus(const FaceState<C>& L, const FaceState<C>& R, C* f) {
    const C alpha = (C)0.1875, beta = (C)0.125;
    C cm = cmax(sound_speed<M>(L.p, L.q[0]), sound_speed<M>(R.p, R.q[0]));
    C icm = M::rcp(cm);
    C mL = L.vel[D] * icm, mR = R.vel[D] * icm;
    C mp, pp, mm, pm;
    if (fabs(mL) >= (C)1.0) {
        mp = (C)0.5 * (mL + fabs(mL));
        pp = mL > (C)0.0 ? (C)1.0 : (C)0.0;
    } else {
        C a = mL + (C)1.0, b = mL * mL - (C)1.0;
        mp = (C)0.25 * a * a + beta * b * b;
        pp = (C)0.25 * a * a * ((C)2.0 - mL) + alpha * mL * b * b;
    }
    if (fabs(mR) >= (C)1.0) {
        mm = (C)0.5 * (mR - fabs(mR));
        pm = mR < (C)0.0 ? (C)1.0 : (C)0.0;
    } else {
        C a = mR - (C)1.0, b = mR * mR - (C)1.0;
        mm = -(C)0.25 * a * a - beta * b * b;
        pm = (C)0.25 * a * a * ((C)2.0 + mR) - alpha * mR * b * b;
    }
    C m = mp + mm;
    C pf = pp * L.p + pm * R.p;
    const bool up = m > (C)0.0;
    const FaceState<C>& W = up ? L : R;
    C mdot = m * cm * W.q[0];
    f[0] = mdot;
    f[1] = mdot * W.vel[0];
    f[2] = mdot * W.vel[1];
    f[3] = mdot * W.vel[2];
    f[1 + D] += pf;
    f[4] = mdot * ((W.q[4] + W.p) * W.ir);
}

template <class M, int D, class C>
__device__ __forceinline__ void slau2(const FaceState<C>& L, const FaceState<C>& R, C* f) {
    C rL = L.q[0], rR = R.q[0];
    C vnL = L.vel[D], vnR = R.vel[D];
    C q2L = L.vel[0] * L.vel[0] + L.vel[1] * L.vel[1] + L.vel[2] * L.vel[2];
    C q2R = R.vel[0] * R.vel[0] + R.vel[1] * R.vel[1] + R.vel[2] * R.vel[2];
    C cf = (C)0.5 * (sound_speed<M>(L.p, rL) + sound_speed<M>(R.p, rR));
    C icf = M::rcp(cf);
    C mL = vnL * icf, mR = vnR * icf;
    C qbar = M::sqrt((C)0.5 * (q2L + q2R));
    C mtil = cmin((C)1.0, icf * qbar);
    C chi = ((C)1.0 - mtil) * ((C)1.0 - mtil);
    C g = -cmax(cmin(mL, (C)0.0), (C)-1.0) * cmin(cmax(mR, (C)0.0), (C)1.0);
    C vbar = M::div(rL * fabs(vnL) + rR * fabs(vnR), rL + rR);
    C vbL = ((C)1.0 - g) * vbar + g * fabs(vnL);
    C vbR = ((C)1.0 - g) * vbar + g * fabs(vnR);
    C mdot = (C)0.5 * (rL * (vnL + vbL) + rR * (vnR - vbR) - (chi * icf) * (R.p - L.p));
    C bL = fabs(mL) < (C)1.0 ? (C)0.25 * ((C)2.0 - mL) * (mL + (C)1.0) * (mL + (C)1.0)
                             : (mL >= (C)0.0 ? (C)1.0 : (C)0.0);
    C bR = fabs(mR) < (C)1.0 ? (C)0.25 * ((C)2.0 + mR) * (mR - (C)1.0) * (mR - (C)1.0)
                             : (mR >= (C)0.0 ? (C)0.0 : (C)1.0);
    C pf = (C)0.5 * (L.p + R.p) + (C)0.5 * (bL - bR) * (L.p - R.p);
    pf += qbar * (bL + bR - (C)1.0) * cf * (C)0.5 * (rL + rR);
    const bool up = mdot > (C)0.0;
    const FaceState<C>& W = up ? L : R;
    f[0] = mdot;
    f[1] = mdot * W.vel[0];
    f[2] = mdot * W.vel[1];
    f[3] = mdot * W.vel[2];
    f[1 + D] += pf;
    f[4] = mdot * ((W.q[4] + W.p) * W.ir);
}

template <class M, int FLUX, int D, class C>
__device__ __forceinline__ void interface_flux(const FaceState<C>& L, const FaceState<C>& R, C* f) {
    if constexpr (FLUX == kSlau2)
        slau2<M, D>(L, R, f);
    else if constexpr (FLUX == kAusmPlus)
        ausm_plus<M, D>(L, R, f);
    else
        rusanov<M, D>(L, R, f);
}

// Scheme chosen at run time (ensembles that mix schemes in one launch).
constexpr int kFluxRuntime = -1;

template <class M, int D, class C>
__device__ __forceinline__ void interface_flux_rt(int flux, const FaceState<C>& L, const FaceState<C>& R, C* f) {
    if (flux == kSlau2)
        slau2<M, D>(L, R, f);
    else if (flux == kAusmPlus)
        ausm_plus<M, D>(L, R, f);
    else
        rusanov<M, D>(L, R, f);
}

}  // namespace od
