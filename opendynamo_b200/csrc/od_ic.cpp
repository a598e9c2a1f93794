// Initial states without Python (declared in include/opendynamo.h):
// od_make_initial_state, the C++ counterpart of the reference's IC
// generator (scripts/make_initial_state.py:122-241) and of this package's
// Taylor-Green state.
//
// The channel and uniform states follow the script's float32 arithmetic
// operation by operation: solution-point coordinates by one double rounding
// of f32 products and sums (the script's math.fma emulation), the laminar
// profile u = 1.5 M (1 - eta^2), rho = 1, p = 1/1.4, and the wall-damped,
// divergence-free Fourier trip whose per-mode wavenumbers, phase and
// amplitudes come from the script's hash fract(sin(s) * 43758.5453). Every
// float operation rounds to float (this file is compiled without
// floating-point contraction), so the trip-free states equal the script's
// bit for bit.
//
// The trip uses float32 sine and cosine. The script takes numpy's, which
// differ from the correctly rounded value in about 15% of arguments; this
// generator takes the correctly rounded one ((float) of the double sine).
// The hash multiplies a one-ulp difference by 4.4e4, so some modes get other
// wavenumbers or phases: the tripped state is a trip of the same kind and
// amplitude, not the script's bits. Runs that must start from the script's
// exact state take its file (or opendynamo_b200.initial_state, which matches
// it bit for bit).

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/opendynamo.h"
#include "od_launch.h"

namespace od {
TablesD host_fr_tables();
}

namespace {

// round_f32(round_f64(a * b + c)) for f32 a, b, c: the f64 product is exact
float fma32(float a, float b, float c) {
    volatile double t = (double)a * (double)b;
    volatile double s = t + (double)c;
    return (float)s;
}

float sin32(float x) { return (float)std::sin((double)x); }
float cos32(float x) { return (float)std::cos((double)x); }

float hash01(float s) {
    volatile float x = sin32(s) * 43758.5453f;
    return x - std::floor(x);
}

struct Points {
    std::vector<float> x, y, z;
};

// centred f32 coordinates of every solution point: fma(L/n, e + 0.5 + 0.5 xi, -L/2)
Points solution_points(int nx, int ny, int nz, float lx, float ly, float lz) {
    const od::TablesD t = od::host_fr_tables();
    float xi[4];
    for (int a = 0; a < 4; ++a) xi[a] = (float)t.pts[a];
    const long long nelem = (long long)nx * ny * nz;
    Points P;
    P.x.resize((size_t)nelem * 64);
    P.y.resize((size_t)nelem * 64);
    P.z.resize((size_t)nelem * 64);
    const float L[3] = {lx, ly, lz};
    const int n[3] = {nx, ny, nz};
    float h[3], shift[3];
    for (int d = 0; d < 3; ++d) {
        volatile float hd = L[d] / (float)n[d];
        volatile float sd = -0.5f * L[d];
        h[d] = hd;
        shift[d] = sd;
    }
    for (long long e = 0; e < nelem; ++e) {
        const long long ex = e % nx, ey = (e / nx) % ny, ez = e / ((long long)nx * ny);
        const float ec[3] = {(float)ex, (float)ey, (float)ez};
        for (int p = 0; p < 64; ++p) {
            const int idx[3] = {p % 4, (p / 4) % 4, p / 16};
            float out[3];
            for (int d = 0; d < 3; ++d) {
                volatile float a = ec[d] + 0.5f;
                volatile float b = 0.5f * xi[idx[d]];
                volatile float mid = a + b;
                out[d] = fma32(h[d], mid, shift[d]);
            }
            const size_t i = (size_t)e * 64 + p;
            P.x[i] = out[0];
            P.y[i] = out[1];
            P.z[i] = out[2];
        }
    }
    return P;
}

// the divergence-free, wall-damped Fourier trip (make_initial_state.py:182-241)
void trip(std::vector<float>* planes, const Points& P, float lx, float ly, float lz, float amplitude, int modes,
          int seed) {
    std::vector<float>& rho = planes[0];
    const size_t np = rho.size();
    const int n_modes = modes > 1 ? modes : 1;
    const float s0 = (float)seed;
    const float half = 0.5f * ly;
    const float weight = amplitude / std::sqrt((float)n_modes);
    const float two_pi = 6.283185307179586f;
    const float mult[6] = {1.113f, 2.229f, 3.717f, 5.381f, 7.993f, 9.677f};
    const float shift[6] = {-3.7183f, 1.7429f, 4.8527f, -2.9956f, 6.1141f, 8.2437f};
    std::vector<float> du(np, 0.0f), dv(np, 0.0f), dw(np, 0.0f);
    std::vector<float> damp(np), damp_y(np);
    for (size_t i = 0; i < np; ++i) {
        volatile float eta = P.y[i] / half;
        volatile float e2 = eta * eta;
        damp[i] = 1.0f - e2;
        volatile float m2 = -2.0f * eta;
        damp_y[i] = m2 / half;
    }
    for (int m = 0; m < n_modes; ++m) {
        volatile float mix = (float)m * 0.113f;
        float r[6];
        for (int q = 0; q < 6; ++q) {
            volatile float prod = mix * mult[q];
            volatile float base = prod + s0;
            volatile float arg = shift[q] < 0.0f ? base - (-shift[q]) : base + shift[q];
            r[q] = hash01(arg);
        }
        volatile float r0 = r[0] * 24.0f, r1 = r[1] * 12.0f;
        const int mx = 1 + (int)r0;
        const int mz = 1 + (int)r1;
        volatile float tkx = two_pi * (float)mx, tkz = two_pi * (float)mz;
        volatile float kx = tkx / lx, kz = tkz / lz;
        volatile float phi = two_pi * r[2];
        volatile float t3 = 2.0f * r[3], t4 = 2.0f * r[4];
        volatile float av = t3 - 1.0f, ac = t4 - 1.0f;
        volatile float wj = 0.5f + r[5];
        volatile float kx2 = kx * kx, kz2 = kz * kz;
        volatile float kh2 = kx2 + kz2;
        const float kh = std::sqrt((float)kh2);
        volatile float ww = weight * wj;
        volatile float wav = ww * av, wac = ww * ac;
        for (size_t i = 0; i < np; ++i) {
            volatile float a = kx * P.x[i], b = kz * P.z[i];
            volatile float ab = a + b;
            volatile float theta = ab + phi;
            const float cos_t = cos32(theta), sin_t = sin32(theta);
            volatile float V = wav * damp[i], Vy = wav * damp_y[i], Cz = wac * damp[i];
            // du += (-1 * (kz * Cz / kh)) * cos_t - (kx * Vy / kh2) * sin_t
            volatile float kzc = kz * Cz;
            volatile float kzck = kzc / kh;
            volatile float nkzck = -1.0f * kzck;
            volatile float t1 = nkzck * cos_t;
            volatile float kxv = kx * Vy;
            volatile float kxvk = kxv / kh2;
            volatile float t2 = kxvk * sin_t;
            volatile float ddu = t1 - t2;
            du[i] = du[i] + ddu;
            volatile float vc = V * cos_t;
            dv[i] = dv[i] + vc;
            // dw += (kx * Cz / kh) * cos_t - (kz * Vy / kh2) * sin_t
            volatile float kxc = kx * Cz;
            volatile float kxck = kxc / kh;
            volatile float w1 = kxck * cos_t;
            volatile float kzv = kz * Vy;
            volatile float kzvk = kzv / kh2;
            volatile float w2 = kzvk * sin_t;
            volatile float ddw = w1 - w2;
            dw[i] = dw[i] + ddw;
        }
    }
    std::vector<float>& m1 = planes[1];
    std::vector<float>& m2 = planes[2];
    std::vector<float>& m3 = planes[3];
    std::vector<float>& E = planes[4];
    for (size_t i = 0; i < np; ++i) {
        volatile float a1 = rho[i] * du[i], a2 = rho[i] * dv[i], a3 = rho[i] * dw[i];
        volatile float n1 = m1[i] + a1, n2 = m2[i] + a2, n3 = m3[i] + a3;
        volatile float q1 = n1 * n1, q2 = n2 * n2, q3 = n3 * n3;
        volatile float s12 = q1 + q2;
        volatile float sn = s12 + q3;
        volatile float o1 = m1[i] * m1[i], o2 = m2[i] * m2[i], o3 = m3[i] * m3[i];
        volatile float o12 = o1 + o2;
        volatile float so = o12 + o3;
        volatile float diff = sn - so;
        volatile float hd = 0.5f * diff;
        volatile float kr = hd / rho[i];
        E[i] = E[i] + kr;
        m1[i] = n1;
        m2[i] = n2;
        m3[i] = n3;
    }
}

}  // namespace

extern "C" int od_make_initial_state(const od_ic_params* p, void* planes, size_t bytes, int u_f64) {
    if (!p || !planes || p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return OD_ERR_ARG;
    if (p->initial_condition < OD_IC_CHANNEL || p->initial_condition > OD_IC_TAYLOR_GREEN) return OD_ERR_ARG;
    const long long nelem = (long long)p->nx * p->ny * p->nz;
    const size_t np = (size_t)nelem * 64;
    if (bytes != np * 5 * (u_f64 ? 8 : 4)) return OD_ERR_SIZE;
    if (p->initial_condition == OD_IC_TAYLOR_GREEN) {
        // u = v0 sin x cos y cos z, v = -v0 cos x sin y cos z, w = 0, rho = 1,
        // p = 1/gamma + v0^2/16 (cos 2x + cos 2y)(cos 2z + 2) on [0, L]^3, in double
        const od::TablesD t = od::host_fr_tables();
        const double v0 = p->mach_bulk, gamma = 1.4;
        const double L[3] = {p->lx, p->ly, p->lz};
        const int n[3] = {p->nx, p->ny, p->nz};
        for (long long e = 0; e < nelem; ++e) {
            const long long ec[3] = {e % p->nx, (e / p->nx) % p->ny, e / ((long long)p->nx * p->ny)};
            for (int q = 0; q < 64; ++q) {
                const int idx[3] = {q % 4, (q / 4) % 4, q / 16};
                double c[3];
                for (int d = 0; d < 3; ++d) c[d] = ((double)ec[d] + 0.5 + 0.5 * t.pts[idx[d]]) * (L[d] / n[d]);
                const double u = v0 * std::sin(c[0]) * std::cos(c[1]) * std::cos(c[2]);
                const double v = -v0 * std::cos(c[0]) * std::sin(c[1]) * std::cos(c[2]);
                const double pr = 1.0 / gamma + v0 * v0 / 16.0 * (std::cos(2 * c[0]) + std::cos(2 * c[1])) *
                                                    (std::cos(2 * c[2]) + 2.0);
                const double E = pr / (gamma - 1.0) + 0.5 * 1.0 * (u * u + v * v);
                const double vals[5] = {1.0, u, v, 0.0, E};
                const size_t i = (size_t)e * 64 + q;
                for (int k = 0; k < 5; ++k) {
                    if (u_f64)
                        static_cast<double*>(planes)[k * np + i] = vals[k];
                    else
                        static_cast<float*>(planes)[k * np + i] = (float)vals[k];
                }
            }
        }
        return OD_OK;
    }
    // the script works on the raw config values: f32 extents, f32 arithmetic
    const float lx = (float)p->lx, ly = (float)p->ly, lz = (float)p->lz;
    const float mach = (float)p->mach_bulk;
    const Points P = solution_points(p->nx, p->ny, p->nz, lx, ly, lz);
    std::vector<float> pl[5];
    for (auto& v : pl) v.assign(np, 0.0f);
    const float pres = 1.0f / 1.4f;
    volatile float gm1v = 1.4f - 1.0f;
    const float gm1 = gm1v;
    volatile float pe = pres / gm1;
    const float half = 0.5f * ly;
    for (size_t i = 0; i < np; ++i) {
        float u;
        if (p->initial_condition == OD_IC_UNIFORM) {
            u = mach;
        } else {
            volatile float eta = P.y[i] / half;
            volatile float prof = fma32(-eta, eta, 1.0f);
            volatile float a = 1.5f * mach;
            u = a * prof;
        }
        pl[0][i] = 1.0f;
        volatile float uu = u * u;
        volatile float ke = 0.5f * 1.0f;
        volatile float ke2 = ke * uu;
        pl[1][i] = 1.0f * u;
        pl[4][i] = pe + ke2;
    }
    if ((float)p->perturbation_amplitude != 0.0f)
        trip(pl, P, lx, ly, lz, (float)p->perturbation_amplitude, p->perturbation_modes, p->perturbation_seed);
    for (int k = 0; k < 5; ++k) {
        if (u_f64) {
            double* dst = static_cast<double*>(planes) + k * np;
            for (size_t i = 0; i < np; ++i) dst[i] = (double)pl[k][i];
        } else {
            std::memcpy(static_cast<float*>(planes) + k * np, pl[k].data(), np * sizeof(float));
        }
    }
    return OD_OK;
}
