// Templated host launcher for one precision combination; included by the
// od_inst_*.cu translation units only.
#pragma once

#include "od_launch.h"
#include "od_stage.cuh"

namespace od {

template <class T>
Tab<T> cast_tab(const TablesD& t) {
    Tab<T> r;
    for (int i = 0; i < 16; ++i) r.D[i] = (T)t.D[i];
    for (int i = 0; i < 4; ++i) {
        r.eL[i] = (T)t.eL[i];
        r.eR[i] = (T)t.eR[i];
        r.gL[i] = (T)t.gL[i];
        r.gR[i] = (T)t.gR[i];
    }
    return r;
}

// The kernels that also write the closure's features exist for the all-f32
// pipeline with constant viscosity at 4 elements per block (the closure's
// configuration); feat says whether this launch writes them.
template <class S, class P, class C, class M>
constexpr bool has_feat_variant() {
    return sizeof(S) == 4 && sizeof(P) == 4 && sizeof(C) == 4 && !M::kSutherland;
}

template <class S, class P, class C, class M, int FLUX, int EPB>
cudaError_t launch_a(const StageAParams<S, P, C>& A, long long nelem, cudaStream_t s, bool feat = false) {
    const unsigned grid = (unsigned)((nelem + EPB - 1) / EPB);
    if (grid == 0) return cudaSuccess;
    const size_t smem = sizeof(SlotA<P, C>) * EPB;
    if constexpr (has_feat_variant<S, P, C, M>() && EPB == 4) {
        if (feat) {
            stage_a_kernel<S, P, C, M, FLUX, EPB, true><<<grid, LPE * EPB, smem, s>>>(A);
            return cudaGetLastError();
        }
    }
    if (feat) return cudaErrorInvalidValue;   // no variant writes the features for this launch
    stage_a_kernel<S, P, C, M, FLUX, EPB><<<grid, LPE * EPB, smem, s>>>(A);
    return cudaGetLastError();
}

template <class S, class P, class C, class M, int FLUX>
cudaError_t launch_a_epb(const StageAParams<S, P, C>& A, long long nelem, int epb, cudaStream_t s, bool feat) {
    if (epb == 2 && !feat) return launch_a<S, P, C, M, FLUX, 2>(A, nelem, s);
    return launch_a<S, P, C, M, FLUX, 4>(A, nelem, s, feat);
}

template <class S, class P, class C, class M>
cudaError_t launch_a_flux(const StageAParams<S, P, C>& A, int flux, long long nelem, int epb, cudaStream_t s,
                          bool feat) {
    if (A.suth >= (C)0) {
        // Sutherland variant: 4 elements per block only, no feature writing
        if (feat) return cudaErrorInvalidValue;
        using MS = WithSutherland<M>;
        switch (flux) {
            case kSlau2: return launch_a<S, P, C, MS, kSlau2, 4>(A, nelem, s);
            case kAusmPlus: return launch_a<S, P, C, MS, kAusmPlus, 4>(A, nelem, s);
            default: return launch_a<S, P, C, MS, kRusanov, 4>(A, nelem, s);
        }
    }
    switch (flux) {
        case kSlau2: return launch_a_epb<S, P, C, M, kSlau2>(A, nelem, epb, s, feat);
        case kAusmPlus: return launch_a_epb<S, P, C, M, kAusmPlus>(A, nelem, epb, s, feat);
        default: return launch_a_epb<S, P, C, M, kRusanov>(A, nelem, epb, s, feat);
    }
}

template <class S, class P, class C, int EPB>
cudaError_t launch_b(const StageBParams<S, P, C>& B, long long nelem, cudaStream_t s) {
    const unsigned grid = (unsigned)((nelem + EPB - 1) / EPB);
    if (grid == 0) return cudaSuccess;
    stage_b_kernel<S, P, C, EPB><<<grid, LPE * EPB, 0, s>>>(B);
    return cudaGetLastError();
}

template <class S, class P, class C, int EPB>
cudaError_t launch_b_split(const StageBParams<S, P, C>& B, long long nelem, cudaStream_t s) {
    const unsigned grid = (unsigned)((nelem + EPB - 1) / EPB);
    if (grid == 0) return cudaSuccess;
    stage_b_split_kernel<S, P, C, EPB><<<grid, LPE * NV * EPB, 0, s>>>(B);
    return cudaGetLastError();
}

// fast math changes only f32 arithmetic: f64-compute combinations use one variant
template <class C>
constexpr bool has_fast_variant() { return sizeof(C) == 4; }

template <class S, class P, class C>
cudaError_t launch_stage_t(const StageLaunch& L, cudaStream_t s) {
    StageAParams<S, P, C> A{};
    A.u_in = (const S*)L.u_in;
    A.u0 = (const S*)L.u0;
    A.u_out = (S*)(L.rhs ? L.rhs : L.u_out);
    A.fv = (C*)L.fv;
    A.fi = (C*)L.fv + L.nelem * kFvWords;
    A.m.nx = L.nx;
    A.m.ny = L.ny;
    A.m.nz = L.nz;
    A.m.y_wall = L.y_wall;
    A.m.nelem = L.nelem;
    mesh_set_div(A.m);
    A.m.npts = L.nelem * NE;
    A.tp = cast_tab<P>(L.tab);
    A.tc = cast_tab<C>(L.tab);
    for (int d = 0; d < 3; ++d) A.jac[d] = (C)L.jac[d];
    A.sc = scale_tab<C>(A.tc, A.jac);
    A.ra = (P)L.ra;
    A.rb = (P)L.rb;
    A.rc = (P)L.rc;
    A.mu = (C)L.mu;
    A.kappa = heat_coeff_host<C>(A.mu);
    A.forcing = (C)L.forcing;
    A.suth = (C)L.suth;
    A.flux = L.flux;
    A.flags = L.flags | (L.rhs ? kDeferRK : 0);
    A.e0 = L.e0;
    A.e1 = L.e1;
    const bool feat = L.feat != nullptr;
    if (feat) A.feat = *L.feat;
    const long long count = L.e1 - L.e0;
    cudaError_t err = cudaSuccess;
    if (L.phases & 1) {
        if (L.ev[0]) cudaEventRecord(L.ev[0], s);
        if constexpr (has_fast_variant<C>()) {
            if (L.fast_math)
                err = launch_a_flux<S, P, C, MathFast>(A, L.flux, count, L.epb_a, s, feat);
            else
                err = launch_a_flux<S, P, C, MathIeee>(A, L.flux, count, L.epb_a, s, feat);
        } else {
            err = launch_a_flux<S, P, C, MathIeee>(A, L.flux, count, L.epb_a, s, feat);
        }
        if (err != cudaSuccess) return err;
        if (L.ev[1]) cudaEventRecord(L.ev[1], s);
    }
    if (L.phases & 2) {
        StageBParams<S, P, C> B;
        B.u_out = (S*)L.u_out;
        B.rhs = (const S*)L.rhs;
        B.u_in = (const S*)L.u_in;
        B.u0 = (const S*)L.u0;
        B.fv = (const C*)L.fv;
        B.fi = A.fi;
        B.m = A.m;
        B.tc = A.tc;
        for (int d = 0; d < 3; ++d) B.jac[d] = A.jac[d];
        B.ra = A.ra;
        B.rb = A.rb;
        B.rc = A.rc;
        B.flags = A.flags;
        B.e0 = L.e0;
        B.e1 = L.e1;
        if (L.epb_b == 8)
            err = launch_b<S, P, C, 8>(B, count, s);
        else if (L.epb_b == 16)
            err = launch_b<S, P, C, 16>(B, count, s);
        else if (L.epb_b == 2)
            err = launch_b_split<S, P, C, 2>(B, count, s);
        else
            err = launch_b_split<S, P, C, 4>(B, count, s);
        if (err != cudaSuccess) return err;
        if (L.ev[2]) cudaEventRecord(L.ev[2], s);
    }
    return cudaSuccess;
}

template <class S, class P, class C, class M, int FLUX>
cudaError_t prepare_flux() {
    cudaError_t e = cudaFuncSetAttribute(stage_a_kernel<S, P, C, M, FLUX, 2>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(sizeof(SlotA<P, C>) * 2));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(stage_a_kernel<S, P, C, WithSutherland<M>, FLUX, 4>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(SlotA<P, C>) * 4));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(stage_a_kernel<S, P, C, M, FLUX, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(SlotA<P, C>) * 4));
}

template <class S, class P, class C, class M>
cudaError_t prepare_m() {
    cudaError_t e = prepare_flux<S, P, C, M, kSlau2>();
    if (e != cudaSuccess) return e;
    e = prepare_flux<S, P, C, M, kAusmPlus>();
    if (e != cudaSuccess) return e;
    return prepare_flux<S, P, C, M, kRusanov>();
}

template <class S, class P, class C>
cudaError_t prepare_t() {
    cudaError_t e = prepare_m<S, P, C, MathIeee>();
    if constexpr (has_fast_variant<C>()) {
        if (e == cudaSuccess) e = prepare_m<S, P, C, MathFast>();
    }
    return e;
}

}  // namespace od

#define OD_INSTANTIATE(NAME, S, P, C)                                                          \
    namespace od {                                                                             \
    cudaError_t launch_stage_##NAME(const StageLaunch& L, cudaStream_t s) {                   \
        return launch_stage_t<S, P, C>(L, s);                                                  \
    }                                                                                          \
    cudaError_t prepare_kernels_##NAME() { return prepare_t<S, P, C>(); }                      \
    }
