// TEST INFRASTRUCTURE ONLY — the CPU oracle for the FR P=3 step path.
//
// A plain C++ restatement of the reference algorithm (drunkseal/opendynamo),
// kept structurally one-to-one with the reference kernels so that every
// intermediate the reference stores (volume RHS, gradient face slices, face
// corrections j, RK stages) can be compared array for array:
//
//   fr_tables()         src/fr_math.rs:3-142 (Gauss-Legendre points, D, extrapolation, Radau g')
//   Phys<C>::pressure   src/cuda/device_functions.cuh:1-5
//   Phys<C>::euler      src/cuda/device_functions.cuh:7-21
//   Phys<C>::viscous    src/cuda/device_functions.cuh:23-102
//   Phys<C>::rusanov    src/cuda/device_functions.cuh:104-128
//   Phys<C>::ausm_plus  src/cuda/device_functions.cuh:130-188
//   Phys<C>::slau2      src/cuda/device_functions.cuh:190-257
//   volume()            src/cuda/rhs.cu:344-511 (gradient, BR1 jumps, wall mirror, Q rounding,
//                       slices rhs.cu:126-180, volume divergence rhs.cu:229-266, forcing rhs.cu:508)
//   faces()             src/cuda/rhs.cu:513-556 (x), 615-687 (y), 572-613 (y wall), 689-739 (z),
//                       compute_face_j rhs.cu:273-297, compute_face_j_wall rhs.cu:311-339
//   rk()                src/cuda/rk.cu:12-115
//   run()               src/solver.rs:262-317 (Shu-Osher SSP-RK3, buffer swap, coefficients)
//
// Nothing in the product links this file: it is loaded only by the tests, by
// __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline leg.
// Precision follows the reference's U/Q/RHS/COMPUTE split: values are loaded
// from the U type into the COMPUTE type C, gradients are rounded through Q,
// the volume RHS is stored in the RHS type, slices and j are stored in C.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int NP = 4;    // points per direction (P = 3)
constexpr int NF = 16;   // points per face
constexpr int NE = 64;   // points per element
constexpr int NV = 5;    // conserved variables

struct Tables {
    double pts[NP], D[NP * NP], eL[NP], eR[NP], gL[NP], gR[NP];
};

// Legendre recurrence (fr_math.rs:3-21).
double legendre(int p, double x) {
    if (p == 0) return 1.0;
    if (p == 1) return x;
    double pm2 = 1.0, pm1 = x, val = 0.0;
    for (int k = 2; k <= p; ++k) {
        double kf = (double)k;
        val = ((2.0 * kf - 1.0) * x * pm1 - (kf - 1.0) * pm2) / kf;
        pm2 = pm1;
        pm1 = val;
    }
    return val;
}

double legendre_deriv(int p, double x) {
    if (p == 0) return 0.0;
    double pf = (double)p;
    return pf / (x * x - 1.0) * (x * legendre(p, x) - legendre(p - 1, x));
}

double lagrange(const double* x, int i, double at) {
    double v = 1.0;
    for (int j = 0; j < NP; ++j)
        if (j != i) v *= (at - x[j]) / (x[i] - x[j]);
    return v;
}

Tables fr_tables() {
    Tables t;
    const int n = NP, p = NP - 1;
    for (int i = 0; i < n; ++i) {
        double x = std::cos(M_PI * ((double)i + 0.75) / ((double)n + 0.5));
        for (;;) {
            double step = legendre(n, x) / legendre_deriv(n, x);
            x -= step;
            if (std::fabs(step) < 1e-14) break;
        }
        t.pts[i] = x;
    }
    std::sort(t.pts, t.pts + n);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            if (i != j) {
                double num = 1.0, den = 1.0;
                for (int k = 0; k < n; ++k) {
                    if (k != i && k != j) num *= t.pts[i] - t.pts[k];
                    if (k != j) den *= t.pts[j] - t.pts[k];
                }
                t.D[i * n + j] = num / den;
            } else {
                double s = 0.0;
                for (int k = 0; k < n; ++k)
                    if (k != i) s += 1.0 / (t.pts[i] - t.pts[k]);
                t.D[i * n + i] = s;
            }
        }
        t.eL[i] = lagrange(t.pts, i, -1.0);
        t.eR[i] = lagrange(t.pts, i, 1.0);
    }
    double sign = (p % 2 == 0) ? 1.0 : -1.0;
    for (int i = 0; i < n; ++i) {
        double dp = legendre_deriv(p, t.pts[i]);
        double dp1 = legendre_deriv(p + 1, t.pts[i]);
        t.gR[i] = 0.5 * (dp + dp1);
        t.gL[i] = 0.5 * sign * (dp - dp1);
    }
    return t;
}

// ---------------------------------------------------------------------------
// Pointwise physics in compute type C.
// ---------------------------------------------------------------------------
template <class C>
struct Phys {
    C mu;
    C suth = (C)-1.0;  // Sutherland S = s_suth / t_ref; < 0: constant mu

    // mu * T^1.5 (1 + S) / (T + S), T = gamma * p / rho with the clamped pressure
    C mu_at(const C* q) const {
        if (suth < (C)0.0) return mu;
        C T = gam * pressure(q) / q[0];
        return mu * T * std::sqrt(T) * ((C)1.0 + suth) / (T + suth);
    }
    const C gam = (C)1.4;
    const C pr = (C)0.72;

    C pressure(const C* q) const {
        C ke = (C)0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / q[0];
        C p = (gam - (C)1.0) * (q[4] - ke);
        return std::max((C)1e-7, p);
    }

    void euler(int d, const C* q, C* f) const {
        C vn = q[1 + d] / q[0];
        C p = pressure(q);
        f[0] = q[1 + d];
        f[1] = q[1] * vn;
        f[2] = q[2] * vn;
        f[3] = q[3] * vn;
        f[1 + d] += p;
        f[4] = vn * (q[4] + p);
    }

    // g[3*var + dir]; the stress/heat-flux algebra of device_functions.cuh:23-102.
    void viscous(int d, const C* q, const C* g, C* f) const {
        const C mu = mu_at(q);
        C r = q[0];
        C vel[3] = {q[1] / r, q[2] / r, q[3] / r};
        // dvel[a][b] = d(vel_a)/d(x_b)
        C dvel[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) dvel[a][b] = (g[3 * (1 + a) + b] - vel[a] * g[b]) / r;
        C div = dvel[0][0] + dvel[1][1] + dvel[2][2];
        C tau[3];
        for (int a = 0; a < 3; ++a) {
            if (a == d)
                tau[a] = mu * ((C)2.0 * dvel[d][d] - (C)2.0 / (C)3.0 * div);
            else
                tau[a] = mu * (dvel[a][d] + dvel[d][a]);
        }
        C ke = (C)0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) / r;
        C p = (gam - (C)1.0) * (q[4] - ke);
        C dke = (q[1] * g[3 + d] + q[2] * g[6 + d] + q[3] * g[9 + d]) / r - ke * g[d] / r;
        C dp = (gam - (C)1.0) * (g[12 + d] - dke);
        C coeff = mu * gam / (pr * (gam - (C)1.0));
        C heat = -coeff * (dp / r - p * g[d] / (r * r));
        f[0] = (C)0.0;
        f[1] = tau[0];
        f[2] = tau[1];
        f[3] = tau[2];
        f[4] = vel[0] * tau[0] + vel[1] * tau[1] + vel[2] * tau[2] - heat;
    }

    C sound(C p, C r) const { return std::sqrt(std::max((C)0.0, gam * p / std::max((C)1e-7, r))); }

    void rusanov(const C* L, const C* R, int d, C* f) const {
        C pL = pressure(L), pR = pressure(R);
        C vnL = L[1 + d] / L[0], vnR = R[1 + d] / R[0];
        C cL = sound(pL, L[0]), cR = sound(pR, R[0]);
        C smax = std::max(std::fabs(vnL) + cL, std::fabs(vnR) + cR);
        C fL[5] = {L[0] * vnL, L[1] * vnL, L[2] * vnL, L[3] * vnL, vnL * (L[4] + pL)};
        C fR[5] = {R[0] * vnR, R[1] * vnR, R[2] * vnR, R[3] * vnR, vnR * (R[4] + pR)};
        fL[1 + d] += pL;
        fR[1 + d] += pR;
        for (int v = 0; v < 5; ++v) f[v] = (C)0.5 * (fL[v] + fR[v] - smax * (R[v] - L[v]));
    }

    void ausm_plus(const C* L, const C* R, int d, C* f) const {
        C pL = pressure(L), pR = pressure(R);
        C uL[3] = {L[1] / L[0], L[2] / L[0], L[3] / L[0]};
        C uR[3] = {R[1] / R[0], R[2] / R[0], R[3] / R[0]};
        C hL = (L[4] + pL) / L[0], hR = (R[4] + pR) / R[0];
        C cmax = std::max(sound(pL, L[0]), sound(pR, R[0]));
        C mL = uL[d] / cmax, mR = uR[d] / cmax;
        const C alpha = (C)0.1875, beta = (C)0.125;
        C mplus, pplus, mminus, pminus;
        if (std::fabs(mL) >= (C)1.0) {
            mplus = (C)0.5 * (mL + std::fabs(mL));
            pplus = mL > (C)0.0 ? (C)1.0 : (C)0.0;
        } else {
            C a = mL + (C)1.0, b = mL * mL - (C)1.0;
            mplus = (C)0.25 * a * a + beta * b * b;
            pplus = (C)0.25 * a * a * ((C)2.0 - mL) + alpha * mL * b * b;
        }
        if (std::fabs(mR) >= (C)1.0) {
            mminus = (C)0.5 * (mR - std::fabs(mR));
            pminus = mR < (C)0.0 ? (C)1.0 : (C)0.0;
        } else {
            C a = mR - (C)1.0, b = mR * mR - (C)1.0;
            mminus = -(C)0.25 * a * a - beta * b * b;
            pminus = (C)0.25 * a * a * ((C)2.0 + mR) - alpha * mR * b * b;
        }
        C m = mplus + mminus;
        C pf = pplus * pL + pminus * pR;
        bool up = m > (C)0.0;
        C mdot = m * cmax * (up ? L[0] : R[0]);
        const C* u = up ? uL : uR;
        f[0] = mdot;
        f[1] = mdot * u[0];
        f[2] = mdot * u[1];
        f[3] = mdot * u[2];
        f[1 + d] += pf;
        f[4] = mdot * (up ? hL : hR);
    }

    void slau2(const C* L, const C* R, int d, C* f) const {
        C rL = L[0], rR = R[0];
        C uL[3] = {L[1] / rL, L[2] / rL, L[3] / rL};
        C uR[3] = {R[1] / rR, R[2] / rR, R[3] / rR};
        C pL = pressure(L), pR = pressure(R);
        C vnL = uL[d], vnR = uR[d];
        C hL = (L[4] + pL) / rL, hR = (R[4] + pR) / rR;
        C q2L = uL[0] * uL[0] + uL[1] * uL[1] + uL[2] * uL[2];
        C q2R = uR[0] * uR[0] + uR[1] * uR[1] + uR[2] * uR[2];
        C cf = (C)0.5 * (sound(pL, rL) + sound(pR, rR));
        C mL = vnL / cf, mR = vnR / cf;
        C qbar = std::sqrt((C)0.5 * (q2L + q2R));
        C mtil = std::min((C)1.0, ((C)1.0 / cf) * qbar);
        C chi = ((C)1.0 - mtil) * ((C)1.0 - mtil);
        C g = -std::max(std::min(mL, (C)0.0), (C)-1.0) * std::min(std::max(mR, (C)0.0), (C)1.0);
        C vbar = (rL * std::fabs(vnL) + rR * std::fabs(vnR)) / (rL + rR);
        C vbL = ((C)1.0 - g) * vbar + g * std::fabs(vnL);
        C vbR = ((C)1.0 - g) * vbar + g * std::fabs(vnR);
        C mdot = (C)0.5 * (rL * (vnL + vbL) + rR * (vnR - vbR) - (chi / cf) * (pR - pL));
        C bL, bR;
        if (std::fabs(mL) < (C)1.0)
            bL = (C)0.25 * ((C)2.0 - mL) * (mL + (C)1.0) * (mL + (C)1.0);
        else
            bL = mL >= (C)0.0 ? (C)1.0 : (C)0.0;
        if (std::fabs(mR) < (C)1.0)
            bR = (C)0.25 * ((C)2.0 + mR) * (mR - (C)1.0) * (mR - (C)1.0);
        else
            bR = mR >= (C)0.0 ? (C)0.0 : (C)1.0;
        C pf = (C)0.5 * (pL + pR) + (C)0.5 * (bL - bR) * (pL - pR);
        pf += qbar * (bL + bR - (C)1.0) * cf * (C)0.5 * (rL + rR);
        bool up = mdot > (C)0.0;
        const C* u = up ? uL : uR;
        f[0] = mdot;
        f[1] = mdot * u[0];
        f[2] = mdot * u[1];
        f[3] = mdot * u[2];
        f[1 + d] += pf;
        f[4] = mdot * (up ? hL : hR);
    }

    void riemann(int scheme, const C* L, const C* R, int d, C* f) const {
        if (scheme == 0)
            slau2(L, R, d, f);
        else if (scheme == 1)
            ausm_plus(L, R, d, f);
        else
            rusanov(L, R, d, f);
    }
};

template <class F>
void parallel_for(long n, int threads, F fn) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (threads == 1 || n < 64) {
        for (long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    long chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        long lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([=, &fn] {
            for (long i = lo; i < hi; ++i) fn(i);
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Parameters of one oracle run. Box extents are the values the reference
// passes to its kernels (f32-rounded config values widened to double).
typedef struct {
    int nx, ny, nz;
    double lx, ly, lz;
    int flux;      // 0 slau2, 1 ausm+, 2 rusanov
    int y_wall;    // 1 slip walls in y, 0 periodic
    int u_f64, q_f64, rhs_f64, c_f64;
    double mu;      // reference: 1.6e-4 (constants.cuh:42)
    double forcing; // reference: 1e-3 on rho*u (rhs.cu:508)
    int threads;    // 0 = all host threads
    int ref_y_slice_f32;  // f64 compute: y slices with f32 products and pair sums, as rhs.cu:145-160
    double suth;          // Sutherland S = s_suth / t_ref (extension); < 0: constant mu as the reference
} orc_params;

}  // extern "C"

namespace {

template <class U, class C>
struct Oracle {
    const orc_params& P;
    Tables T;
    C pts[NP], D[NP * NP], eL[NP], eR[NP], gL[NP], gR[NP];
    Phys<C> ph;
    long nelem, npts;
    C jac[3];

    explicit Oracle(const orc_params& p) : P(p) {
        T = fr_tables();
        for (int i = 0; i < NP; ++i) {
            pts[i] = (C)T.pts[i];
            eL[i] = (C)T.eL[i];
            eR[i] = (C)T.eR[i];
            gL[i] = (C)T.gL[i];
            gR[i] = (C)T.gR[i];
        }
        for (int i = 0; i < NP * NP; ++i) D[i] = (C)T.D[i];
        ph.mu = (C)p.mu;
        ph.suth = (C)p.suth;
        nelem = (long)p.nx * p.ny * p.nz;
        npts = nelem * NE;
        C L[3] = {(C)p.lx, (C)p.ly, (C)p.lz};
        int n[3] = {p.nx, p.ny, p.nz};
        for (int d = 0; d < 3; ++d) jac[d] = (C)2.0 / (L[d] / (C)n[d]);
    }

    C qround(C x) const { return (P.q_f64 || sizeof(C) == 4) ? x : (C)(float)x; }

    long elem_id(int ex, int ey, int ez) const { return ex + (long)P.nx * (ey + (long)P.ny * ez); }

    // point index of (i, j, k) inside an element
    static int pid(int i, int j, int k) { return i + NP * j + NF * k; }

    // point of line `line` (the two non-d coordinates as a face point) at position m along d
    static int line_pt(int d, int fp, int m) {
        int a = fp % NP, b = fp / NP;
        if (d == 0) return pid(m, a, b);  // face pt = j + 4k
        if (d == 1) return pid(a, m, b);  // face pt = i + 4k
        return pid(a, b, m);              // face pt = i + 4j
    }
    static int face_pt(int d, int pt) {
        int i = pt % NP, j = (pt / NP) % NP, k = pt / NF;
        if (d == 0) return j + NP * k;
        if (d == 1) return i + NP * k;
        return i + NP * j;
    }
    static int along(int d, int pt) {
        int i = pt % NP, j = (pt / NP) % NP, k = pt / NF;
        return d == 0 ? i : (d == 1 ? j : k);
    }

    void load_elem(const U* u, long e, C out[NV][NE]) const {
        for (int v = 0; v < NV; ++v)
            for (int p = 0; p < NE; ++p) out[v][p] = (C)u[v * npts + e * NE + p];
    }

    // neighbour of element (ex,ey,ez) in direction d, side s (0 = minus, 1 = plus);
    // returns -1 for a y wall.
    long neighbour(int ex, int ey, int ez, int d, int s) const {
        int c[3] = {ex, ey, ez};
        int n[3] = {P.nx, P.ny, P.nz};
        int t = c[d] + (s ? 1 : -1);
        if (d == 1 && P.y_wall && (t < 0 || t >= n[1])) return -1;
        c[d] = (t + n[d]) % n[d];
        return elem_id(c[0], c[1], c[2]);
    }

    // slice row: which of the 15 gradient components each direction keeps (rhs.cu:129,151,169)
    static bool omitted(int d, int c) {
        static const int om[3][4] = {{8, 10, 13, 14}, {5, 9, 12, 14}, {4, 6, 12, 13}};
        for (int q = 0; q < 4; ++q)
            if (om[d][q] == c) return true;
        return false;
    }

    // ----- compute_rhs_volume_kernel -----
    template <class R>
    void volume(const U* u, R* rhs, C* slices[6]) const {
        parallel_for(nelem, P.threads, [&](long e) {
            int ex = (int)(e % P.nx), ey = (int)((e / P.nx) % P.ny), ez = (int)(e / ((long)P.nx * P.ny));
            C q[NV][NE];
            load_elem(u, e, q);
            C grad[15][NE];
            for (int p = 0; p < NE; ++p)
                for (int v = 0; v < NV; ++v)
                    for (int d = 0; d < 3; ++d) {
                        C s = 0;
                        int a = along(d, p), fp = face_pt(d, p);
                        for (int m = 0; m < NP; ++m) s += D[a * NP + m] * q[v][line_pt(d, fp, m)];
                        grad[3 * v + d][p] = s * jac[d];
                    }
            // BR1 jumps with the six neighbours' face values
            for (int d = 0; d < 3; ++d) {
                for (int side = 0; side < 2; ++side) {
                    long nb = neighbour(ex, ey, ez, d, side);
                    C qn[NV][NE];
                    if (nb >= 0) load_elem(u, nb, qn);
                    const C* own_c = side ? eR : eL;   // own trace at this side
                    const C* nb_c = side ? eL : eR;    // neighbour trace at the opposite side
                    const C* gp = side ? gR : gL;
                    for (int fp = 0; fp < NF; ++fp)
                        for (int v = 0; v < NV; ++v) {
                            C own = 0, other = 0;
                            for (int m = 0; m < NP; ++m) own += q[v][line_pt(d, fp, m)] * own_c[m];
                            if (nb >= 0) {
                                for (int m = 0; m < NP; ++m) other += qn[v][line_pt(d, fp, m)] * nb_c[m];
                            } else {
                                other = (v > 0 && v < 4) ? -own : own;  // reflect_wall
                            }
                            C jump = (C)0.5 * (other + own) - own;
                            for (int m = 0; m < NP; ++m) grad[3 * v + d][line_pt(d, fp, m)] += jump * gp[m] * jac[d];
                        }
                }
            }
            for (int c = 0; c < 15; ++c)
                for (int p = 0; p < NE; ++p) grad[c][p] = qround(grad[c][p]);
            // gradient face slices
            for (int d = 0; d < 3; ++d)
                for (int fp = 0; fp < NF; ++fp) {
                    C* rowL = slices[2 * d] + ((size_t)e * NF + fp) * 12;
                    C* rowR = slices[2 * d + 1] + ((size_t)e * NF + fp) * 12;
                    int slot = 0;
                    for (int c = 0; c < 15; ++c) {
                        if (omitted(d, c)) continue;
                        C sl = 0, sr = 0;
                        if (d == 1 && (P.ref_y_slice_f32 || sizeof(C) == 4)) {
                            // rhs.cu:157-160: __fmul_rn products, (p0 + p1) + (p2 + p3) in f32
                            float pl[4], pr[4];
                            for (int m = 0; m < NP; ++m) {
                                pl[m] = (float)grad[c][line_pt(d, fp, m)] * (float)eL[m];
                                pr[m] = (float)grad[c][line_pt(d, fp, m)] * (float)eR[m];
                            }
                            sl = (C)((pl[0] + pl[1]) + (pl[2] + pl[3]));
                            sr = (C)((pr[0] + pr[1]) + (pr[2] + pr[3]));
                        } else {
                            for (int m = 0; m < NP; ++m) {
                                sl += grad[c][line_pt(d, fp, m)] * eL[m];
                                sr += grad[c][line_pt(d, fp, m)] * eR[m];
                            }
                        }
                        rowL[slot] = sl;
                        rowR[slot] = sr;
                        ++slot;
                    }
                    rowL[11] = 0;
                    rowR[11] = 0;
                }
            // volume divergence of (F_euler - F_viscous)
            C flux[3][NV][NE];
            for (int p = 0; p < NE; ++p) {
                C qs[NV], gs[15];
                for (int v = 0; v < NV; ++v) qs[v] = q[v][p];
                for (int c = 0; c < 15; ++c) gs[c] = grad[c][p];
                for (int d = 0; d < 3; ++d) {
                    C fe[NV], fv[NV];
                    ph.euler(d, qs, fe);
                    ph.viscous(d, qs, gs, fv);
                    for (int v = 0; v < NV; ++v) flux[d][v][p] = fe[v] - fv[v];
                }
            }
            for (int p = 0; p < NE; ++p)
                for (int v = 0; v < NV; ++v) {
                    C sum = 0;
                    for (int d = 0; d < 3; ++d) {
                        int a = along(d, p), fp = face_pt(d, p);
                        C df = 0;
                        for (int m = 0; m < NP; ++m) df += D[a * NP + m] * flux[d][v][line_pt(d, fp, m)];
                        sum += df * jac[d];
                    }
                    C r = -sum;
                    if (v == 1) r += (C)P.forcing;
                    rhs[v * npts + e * NE + p] = (R)r;
                }
        });
    }

    void unpack_slice(int d, const C* row, C* g) const {
        int slot = 0;
        for (int c = 0; c < 15; ++c) {
            if (omitted(d, c)) {
                g[c] = 0;
                continue;
            }
            g[c] = row[slot++];
        }
    }

    // face value of element e at direction d, side s, face point fp
    void trace(const U* u, long e, int d, int s, int fp, C* out) const {
        const C* c = s ? eR : eL;
        for (int v = 0; v < NV; ++v) {
            C acc = 0;
            for (int m = 0; m < NP; ++m) acc += (C)u[v * npts + e * NE + line_pt(d, fp, m)] * c[m];
            out[v] = acc;
        }
    }

    // ----- compute_face_flux_{x,y,z}_kernel + compute_face_flux_y_wall_kernel -----
    void faces(const U* u, C* const slices[6], C* j[6]) const {
        long nf = nelem * NF;
        parallel_for(nelem, P.threads, [&](long e) {
            int ex = (int)(e % P.nx), ey = (int)((e / P.nx) % P.ny), ez = (int)(e / ((long)P.nx * P.ny));
            for (int d = 0; d < 3; ++d) {
                // the face on the minus side of element e (e is the right element)
                long left = neighbour(ex, ey, ez, d, 0);
                for (int fp = 0; fp < NF; ++fp) {
                    if (left >= 0) {
                        C uL[NV], uR[NV], gLf[15], gRf[15];
                        trace(u, left, d, 1, fp, uL);
                        trace(u, e, d, 0, fp, uR);
                        unpack_slice(d, slices[2 * d + 1] + ((size_t)left * NF + fp) * 12, gLf);
                        unpack_slice(d, slices[2 * d] + ((size_t)e * NF + fp) * 12, gRf);
                        C fi[NV], fvL[NV], fvR[NV], feL[NV], feR[NV];
                        ph.riemann(P.flux, uL, uR, d, fi);
                        ph.viscous(d, uL, gLf, fvL);
                        ph.viscous(d, uR, gRf, fvR);
                        ph.euler(d, uL, feL);
                        ph.euler(d, uR, feR);
                        for (int v = 0; v < NV; ++v) {
                            C fc = fi[v] - (C)0.5 * (fvL[v] + fvR[v]);
                            j[2 * d + 1][v * nf + left * NF + fp] = fc - (feL[v] - fvL[v]);
                            j[2 * d][v * nf + e * NF + fp] = fc - (feR[v] - fvR[v]);
                        }
                    } else {
                        wall_face(u, slices, j, e, 0, fp);
                    }
                }
                if (d == 1 && P.y_wall && ey == P.ny - 1) {
                    for (int fp = 0; fp < NF; ++fp) wall_face(u, slices, j, e, 1, fp);
                }
            }
        });
    }

    // slip wall: flux [0, 0, p_wall, 0, 0], viscous traction = own (rhs.cu:311-339)
    void wall_face(const U* u, C* const slices[6], C* j[6], long e, int upper, int fp) const {
        long nf = nelem * NF;
        C q[NV], g[15];
        trace(u, e, 1, upper, fp, q);
        unpack_slice(1, slices[2 + upper] + ((size_t)e * NF + fp) * 12, g);
        C fv[NV], fe[NV];
        ph.viscous(1, q, g, fv);
        ph.euler(1, q, fe);
        C v2r = q[2] * q[2] / q[0];
        C fw[NV] = {0, 0, fe[2] - v2r, 0, 0};
        for (int v = 0; v < NV; ++v) {
            C fc = fw[v] - fv[v];
            j[2 + upper][v * nf + e * NF + fp] = fc - (fe[v] - fv[v]);
        }
    }

    // volume RHS plus the lifted face corrections, in C (rk.cu:12-25)
    template <class R>
    C total(const R* rhs, C* const j[6], long e, int p, int v) const {
        long nf = nelem * NF;
        C r = (C)rhs[v * npts + e * NE + p];
        C corr[3];
        for (int d = 0; d < 3; ++d) {
            int a = along(d, p), fp = face_pt(d, p);
            C jl = j[2 * d][v * nf + e * NF + fp], jr = j[2 * d + 1][v * nf + e * NF + fp];
            corr[d] = -(jl * gL[a] * jac[d]) - (jr * gR[a] * jac[d]);
        }
        return r + (corr[0] + corr[1] + corr[2]);
    }

    // ----- rk_stage_kernel / rk_stage1_kernel -----
    template <class R>
    void rk(U* dst, const U* src, const R* rhs, C* const j[6], C a, C b, C c, bool stage1) const {
        parallel_for(nelem, P.threads, [&](long e) {
            for (int v = 0; v < NV; ++v)
                for (int p = 0; p < NE; ++p) {
                    long idx = v * npts + e * NE + p;
                    C t = total(rhs, j, e, p, v);
                    C out = stage1 ? a * (C)src[idx] + c * t : a * (C)src[idx] + b * (C)dst[idx] + c * t;
                    dst[idx] = (U)out;
                }
        });
    }
};

template <class U, class C, class R>
struct Buffers {
    std::vector<R> rhs;
    std::vector<C> sl[6], jj[6];
    C* slp[6];
    C* jp[6];
    Buffers(long nelem) : rhs(nelem * NE * NV) {
        for (int q = 0; q < 6; ++q) {
            sl[q].assign(nelem * NF * 12, 0);
            jj[q].assign(nelem * NF * NV, 0);
            slp[q] = sl[q].data();
            jp[q] = jj[q].data();
        }
    }
};

template <class U, class C, class R>
void run_impl(const orc_params& p, U* u, int n_steps, double dt_in) {
    Oracle<U, C> o(p);
    Buffers<U, C, R> b(o.nelem);
    std::vector<U> uprev(o.npts * NV);
    U* cur = u;
    U* prev = uprev.data();
    C dt = (C)dt_in;
    for (int s = 0; s < n_steps; ++s) {
        o.volume(cur, b.rhs.data(), b.slp);
        o.faces(cur, b.slp, b.jp);
        o.rk(prev, cur, b.rhs.data(), b.jp, (C)1.0, (C)0.0, dt, true);
        std::swap(cur, prev);
        o.volume(cur, b.rhs.data(), b.slp);
        o.faces(cur, b.slp, b.jp);
        o.rk(cur, prev, b.rhs.data(), b.jp, (C)0.75, (C)0.25, (C)0.25 * dt, false);
        o.volume(cur, b.rhs.data(), b.slp);
        o.faces(cur, b.slp, b.jp);
        o.rk(cur, prev, b.rhs.data(), b.jp, (C)(1.0 / 3.0), (C)(2.0 / 3.0), (C)(2.0 / 3.0) * dt, false);
    }
    if (cur != u) std::memcpy(u, cur, sizeof(U) * o.npts * NV);
}

// Runtime dispatch over the U / C / RHS storage types.
template <template <class, class, class> class Fn, class... A>
int dispatch(const orc_params& p, A... args) {
    if (p.u_f64) {
        if (p.c_f64) {
            if (p.rhs_f64) return Fn<double, double, double>::go(p, args...);
            return Fn<double, double, float>::go(p, args...);
        }
        if (p.rhs_f64) return Fn<double, float, double>::go(p, args...);
        return Fn<double, float, float>::go(p, args...);
    }
    if (p.c_f64) {
        if (p.rhs_f64) return Fn<float, double, double>::go(p, args...);
        return Fn<float, double, float>::go(p, args...);
    }
    if (p.rhs_f64) return Fn<float, float, double>::go(p, args...);
    return Fn<float, float, float>::go(p, args...);
}

template <class U, class C, class R>
struct VolumeFn {
    static int go(const orc_params& p, const void* u, void* rhs, void** sl) {
        Oracle<U, C> o(p);
        C* s[6];
        for (int q = 0; q < 6; ++q) s[q] = (C*)sl[q];
        o.volume((const U*)u, (R*)rhs, s);
        return 0;
    }
};

template <class U, class C, class R>
struct FacesFn {
    static int go(const orc_params& p, const void* u, void** sl, void** j) {
        Oracle<U, C> o(p);
        C* s[6];
        C* jj[6];
        for (int q = 0; q < 6; ++q) {
            s[q] = (C*)sl[q];
            jj[q] = (C*)j[q];
        }
        o.faces((const U*)u, s, jj);
        return 0;
    }
};

template <class U, class C, class R>
struct RkFn {
    static int go(const orc_params& p, void* dst, const void* src, const void* rhs, void** j, double a, double b,
                  double c, int stage1) {
        Oracle<U, C> o(p);
        C* jj[6];
        for (int q = 0; q < 6; ++q) jj[q] = (C*)j[q];
        o.rk((U*)dst, (const U*)src, (const R*)rhs, jj, (C)a, (C)b, (C)c, stage1 != 0);
        return 0;
    }
};

template <class U, class C, class R>
struct TotalFn {
    static int go(const orc_params& p, const void* u, double* out) {
        Oracle<U, C> o(p);
        Buffers<U, C, R> b(o.nelem);
        o.volume((const U*)u, b.rhs.data(), b.slp);
        o.faces((const U*)u, b.slp, b.jp);
        parallel_for(o.nelem, p.threads, [&](long e) {
            for (int v = 0; v < NV; ++v)
                for (int q = 0; q < NE; ++q) out[v * o.npts + e * NE + q] = (double)o.total(b.rhs.data(), b.jp, e, q, v);
        });
        return 0;
    }
};

template <class U, class C, class R>
struct RunFn {
    static int go(const orc_params& p, void* u, int n, double dt) {
        run_impl<U, C, R>(p, (U*)u, n, dt);
        return 0;
    }
};

bool valid(const orc_params* p) {
    return p && p->nx > 0 && p->ny > 0 && p->nz > 0 && p->flux >= 0 && p->flux <= 2;
}

}  // namespace

extern "C" {

// FR operator tables in double: pts[4], D[16] (row-major, D[i*4+j] = l'_j(x_i)),
// extrap_left[4], extrap_right[4], g_left'[4], g_right'[4].
int orc_fr_tables(double* out36) {
    Tables t = fr_tables();
    std::memcpy(out36, t.pts, 4 * sizeof(double));
    std::memcpy(out36 + 4, t.D, 16 * sizeof(double));
    std::memcpy(out36 + 20, t.eL, 4 * sizeof(double));
    std::memcpy(out36 + 24, t.eR, 4 * sizeof(double));
    std::memcpy(out36 + 28, t.gL, 4 * sizeof(double));
    std::memcpy(out36 + 32, t.gR, 4 * sizeof(double));
    return 0;
}

// Pointwise physics in double (unit tests of the flux functions).
int orc_euler_flux(int d, const double* q, double* f) {
    Phys<double> ph;
    ph.mu = 1.6e-4;
    ph.euler(d, q, f);
    return 0;
}
int orc_viscous_flux(int d, double mu, const double* q, const double* g, double* f) {
    Phys<double> ph;
    ph.mu = mu;
    ph.viscous(d, q, g, f);
    return 0;
}
// Same with Sutherland's law (suth = s_suth / t_ref; < 0: constant mu).
int orc_viscous_flux_suth(int d, double mu, double suth, const double* q, const double* g, double* f) {
    Phys<double> ph;
    ph.mu = mu;
    ph.suth = suth;
    ph.viscous(d, q, g, f);
    return 0;
}
int orc_riemann_flux(int scheme, int d, const double* L, const double* R, double* f) {
    Phys<double> ph;
    ph.mu = 1.6e-4;
    ph.riemann(scheme, L, R, d, f);
    return 0;
}

// compute_rhs_volume_kernel: U (U type) -> RHS (RHS type), 6 slices (C type,
// order x_left, x_right, y_left, y_right, z_left, z_right).
int orc_volume(const orc_params* p, const void* u, void* rhs, void** slices) {
    if (!valid(p)) return -1;
    return dispatch<VolumeFn>(*p, u, rhs, slices);
}

// The three face kernels (+ the wall kernel in wall mode): U + slices -> 6 j arrays (C type).
int orc_faces(const orc_params* p, const void* u, void** slices, void** j) {
    if (!valid(p)) return -1;
    return dispatch<FacesFn>(*p, u, slices, j);
}

// rk_stage1_kernel (stage1 = 1: dst = a*src + c*total) or rk_stage_kernel
// (dst = a*src + b*dst + c*total), in C.
int orc_rk(const orc_params* p, void* dst, const void* src, const void* rhs, void** j, double a, double b, double c,
           int stage1) {
    if (!valid(p)) return -1;
    return dispatch<RkFn>(*p, dst, src, rhs, j, a, b, c, stage1);
}

// Full right-hand side (volume RHS + lifted face corrections) as double.
int orc_rhs_total(const orc_params* p, const void* u, double* out) {
    if (!valid(p)) return -1;
    return dispatch<TotalFn>(*p, u, out);
}

// n SSP-RK3 steps in place on u (U type). dt is used as given (the reference
// rounds the configured dt to f32 first).
int orc_run(const orc_params* p, void* u, int n_steps, double dt) {
    if (!valid(p) || n_steps < 0) return -1;
    return dispatch<RunFn>(*p, u, n_steps, dt);
}

// The same run in extended precision (x87 long double state and arithmetic),
// a more accurate truth for judging f64 implementations. u is double in / out.
int orc_run_ld(const orc_params* p, double* u, int n_steps, double dt) {
    if (!valid(p) || n_steps < 0) return -1;
    long n = (long)p->nx * p->ny * p->nz * NE * NV;
    std::vector<long double> w(u, u + n);
    run_impl<long double, long double, long double>(*p, w.data(), n_steps, dt);
    for (long i = 0; i < n; ++i) u[i] = (double)w[i];
    return 0;
}

}  // extern "C"
