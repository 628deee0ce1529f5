// Device helpers shared by the sweep kernels (ie_kernels.cu, ie_level.cu):
// the steps of a launch, the exchange-phase count and the f32 / exact f64
// forms of the reference's fast_exp acceptance test.
#pragma once
#include <cstdint>

#include "ie_device.cuh"
#include "ie_kernels.cuh"

namespace ie {

// Number of exchange phases executed in global steps (base, base + steps].
__device__ __forceinline__ uint32_t exchanges_in(uint64_t base, uint32_t steps, uint32_t k) {
    return (uint32_t)((base + steps) / k - base / k);
}

// The steps one instance runs in a batched launch: the launch's own schedule,
// or in a serving launch the instance's schedule from its next unexecuted
// step, for the host's plan of the tick or else at most max(1, site_budget /
// unit) steps, unit = the sites of the work item the instance is in (n for
// the per-lane kernels). Step s of the
// launch is global step base + s of the instance and runs at temperature
// temps[tstride * s].
struct StepPlan {
    uint64_t base;
    uint32_t steps;
    uint32_t tstride;
    const double* temps;
};

__device__ __forceinline__ StepPlan step_plan(const DevArrays& A, const RunArgs& R, const InstDesc& d,
                                              uint32_t inst, uint32_t unit = 0) {
    StepPlan P;
    if (R.serve) {
        P.base = A.done[d.owner];
        const uint64_t left = d.sched_len > P.base ? d.sched_len - P.base : 0;
        const uint64_t want = R.plan ? (uint64_t)R.plan[inst] : max(1u, R.site_budget / max(unit ? unit : d.n, 1u));
        P.steps = (uint32_t)min(left, want);
        P.tstride = 1;
        P.temps = R.temps + d.sched + P.base;
    } else {
        P.base = R.step_base_dev ? *R.step_base_dev : R.step_base;
        P.steps = R.steps;
        P.tstride = R.temps_per_step ? (R.cells ? R.ladder : 1u) : 0u;
        P.temps = R.temps + (R.cells ? d.cell : 0u);
    }
    return P;
}

// f32 evaluation of fast_exp, every operation rounded separately (no fused
// multiply-add), used only to pre-decide u < fast_exp(x) outside a relative
// band of 2^-10 around the f64 value; the worst relative gap between this and
// the f64 evaluation over [-20, 0] is below 6e-6.
__device__ __forceinline__ float fast_exp_f32(float x) {
    x = fminf(fmaxf(x, -20.0f), 0.0f);
    const float r = __fmul_rn(x, 0.0625f);
    const float r2 = __fmul_rn(r, r);
    const float r3 = __fmul_rn(r2, r);
    float p = __fadd_rn(1.0f, r);
    p = __fadd_rn(p, __fmul_rn(0.5f, r2));
    p = __fadd_rn(p, __fmul_rn(1.0f / 6.0f, r3));
    p = __fadd_rn(p, __fmul_rn(__fmul_rn(1.0f / 24.0f, r2), r2));
    p = __fadd_rn(p, __fmul_rn(__fmul_rn(1.0f / 120.0f, r2), r3));
    p = __fadd_rn(p, __fmul_rn(__fmul_rn(1.0f / 720.0f, r3), r3));
    const float p2 = __fmul_rn(p, p);
    const float p4 = __fmul_rn(p2, p2);
    const float p8 = __fmul_rn(p4, p4);
    return __fmul_rn(p8, p8);
}

// Exact f64 decision, out of line: only reached inside the f32 band.
static __device__ __noinline__ bool metropolis_exact_f64(double x, uint64_t m) {
    return __dmul_rn((double)m, 2.220446049250313e-16) < fast_exp_rn(x);
}

}  // namespace ie
