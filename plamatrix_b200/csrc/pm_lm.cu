// Levenberg-Marquardt damping strategy and the robust cost of a set of residuals: the caller
// side of the normal-equation path (include/plamatrix/optimization/levenberg_marquardt.h:13-95,
// include/plamatrix/optimization/robust_loss.h:27-51).
//
// The strategy is host state, as in the reference: the caller evaluates the cost of a trial step
// and reports acceptance or rejection.  The cost is evaluated on the device, so an LM loop over
// device-resident residuals needs one scalar read per trial step.  Each observation's Huber cost
// is evaluated in the residual's scalar type exactly as evaluateHuberLoss does; the costs are
// summed in FP64 in a fixed tree (thread-strided runs, then block order), so repeated calls are
// bitwise identical.
#include "pm_common.cuh"

#include <algorithm>
#include <cmath>

struct pm_lm_strategy
{
    int value_size = 8;
    pm_lm_options options{};
    double damping = 0.0;
    int accepted = 0;
    int rejected = 0;
};

namespace pm
{
namespace
{

constexpr int kCostThreads = 256;

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// one block-level partial per block of the launch (kernel 1), then their sum (kernel 2)
template <typename T>
__global__ void __launch_bounds__(kCostThreads) huber_cost_partials_kernel(int64_t count, int m,
                                                                           const T* __restrict__ res, T delta,
                                                                           double* __restrict__ partials)
{
    __shared__ double smem[kCostThreads / 32];
    double mine = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * kCostThreads + threadIdx.x; i < count;
         i += int64_t(gridDim.x) * kCostThreads)
    {
        const T* r = res + i * m;
        T squared = T(0);
        for (int k = 0; k < m; ++k)
            squared = add_rn(squared, mul_rn(r[k], r[k]));
        // evaluateHuberLoss: 0.5 s inside delta, delta sqrt(s) - 0.5 delta^2 outside (each
        // operation rounded on its own, as the host code does)
        T cost;
        if (delta == T(0) || squared <= mul_rn(delta, delta))
            cost = mul_rn(T(0.5), squared);
        else
            cost = sub_rn(mul_rn(delta, sqrt(squared)), mul_rn(mul_rn(T(0.5), delta), delta));
        mine += static_cast<double>(cost);
    }
    const double total = block_sum<double, kCostThreads>(mine, smem);
    if (threadIdx.x == 0)
        partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kCostThreads) huber_cost_finish_kernel(int parts,
                                                                         const double* __restrict__ partials,
                                                                         double* __restrict__ cost)
{
    __shared__ double smem[kCostThreads / 32];
    double mine = 0.0;
    for (int b = threadIdx.x; b < parts; b += kCostThreads)
        mine += partials[b];
    const double total = block_sum<double, kCostThreads>(mine, smem);
    if (threadIdx.x == 0)
        *cost = total;
}

template <typename T>
void huber_cost(cudaStream_t stream, int64_t count, int64_t m, const T* res, T delta, double* scratch, double* cost)
{
    if (count < 0 || m <= 0 || m > 64)
        fail(PM_INVALID_ARGUMENT, "observation count must be non-negative and residual size in [1, 64]");
    if (!std::isfinite(static_cast<double>(delta)) || delta < T(0))
        fail(PM_INVALID_ARGUMENT, "evaluateHuberLoss: delta must be finite and non-negative");
    if (!cost || !scratch || (count > 0 && !res))
        fail(PM_INVALID_ARGUMENT, "Huber cost: residual, scratch and cost pointers must be non-null");
    const unsigned grid = grid_for(count, kCostThreads, PM_HUBER_COST_SCRATCH);
    huber_cost_partials_kernel<T><<<grid, kCostThreads, 0, stream>>>(count, static_cast<int>(m), res, delta, scratch);
    PM_LAUNCH_CHECK();
    huber_cost_finish_kernel<<<1, kCostThreads, 0, stream>>>(static_cast<int>(grid), scratch, cost);
    PM_LAUNCH_CHECK();
}

// the reference's arithmetic in the strategy's scalar type
template <typename T>
void lm_update(pm_lm_strategy* s, bool accept)
{
    const T d = static_cast<T>(s->damping);
    if (accept)
    {
        const T next = d * static_cast<T>(s->options.decrease_factor);
        s->damping = std::max(static_cast<T>(s->options.minimum_damping), next);
        ++s->accepted;
    }
    else
    {
        const T next = d * static_cast<T>(s->options.increase_factor);
        s->damping = std::min(static_cast<T>(s->options.maximum_damping), next);
        ++s->rejected;
    }
}

template <typename T>
void lm_create(const pm_lm_options* o, pm_lm_strategy** out)
{
    if (!out)
        fail(PM_INVALID_ARGUMENT, "output handle pointer is null");
    pm_lm_options opt{};
    if (o)
        opt = *o;
    else
        pm_lm_options_default(&opt);
    const T mn = static_cast<T>(opt.minimum_damping), mx = static_cast<T>(opt.maximum_damping),
            in = static_cast<T>(opt.initial_damping), dec = static_cast<T>(opt.decrease_factor),
            inc = static_cast<T>(opt.increase_factor);
    if (!std::isfinite(mn) || !std::isfinite(mx) || !std::isfinite(in) || mn <= T(0) || mx < mn || in < mn ||
        in > mx || !std::isfinite(dec) || dec <= T(0) || dec >= T(1) || !std::isfinite(inc) || inc <= T(1))
        fail(PM_INVALID_ARGUMENT, "LevenbergMarquardtStrategy: invalid damping options");
    auto* s = new pm_lm_strategy;
    s->value_size = sizeof(T);
    s->options = opt;
    s->damping = static_cast<double>(in);
    *out = s;
}

} // namespace
} // namespace pm

extern "C" {

void pm_lm_options_default(pm_lm_options* o)
{
    if (!o)
        return;
    o->initial_damping = 1e-3;
    o->minimum_damping = 1e-12;
    o->maximum_damping = 1e12;
    o->decrease_factor = 0.3;
    o->increase_factor = 10.0;
}

int pm_lm_strategy_create_f32(const pm_lm_options* options, pm_lm_strategy** out)
{
    return pm::guarded([&] { pm::lm_create<float>(options, out); });
}

int pm_lm_strategy_create_f64(const pm_lm_options* options, pm_lm_strategy** out)
{
    return pm::guarded([&] { pm::lm_create<double>(options, out); });
}

void pm_lm_strategy_destroy(pm_lm_strategy* s) { delete s; }

int pm_lm_accept_step(pm_lm_strategy* s)
{
    return pm::guarded([&] {
        if (!s)
            pm::fail(PM_INVALID_ARGUMENT, "LM strategy handle is null");
        if (s->value_size == 4)
            pm::lm_update<float>(s, true);
        else
            pm::lm_update<double>(s, true);
    });
}

int pm_lm_reject_step(pm_lm_strategy* s)
{
    return pm::guarded([&] {
        if (!s)
            pm::fail(PM_INVALID_ARGUMENT, "LM strategy handle is null");
        if (s->value_size == 4)
            pm::lm_update<float>(s, false);
        else
            pm::lm_update<double>(s, false);
    });
}

int pm_lm_strategy_state(const pm_lm_strategy* s, double* damping, int* accepted_steps, int* rejected_steps)
{
    return pm::guarded([&] {
        if (!s)
            pm::fail(PM_INVALID_ARGUMENT, "LM strategy handle is null");
        if (damping)
            *damping = s->damping;
        if (accepted_steps)
            *accepted_steps = s->accepted;
        if (rejected_steps)
            *rejected_steps = s->rejected;
    });
}

int pm_huber_cost_f32(pm_stream_t stream, int64_t count, int64_t m, const float* residual_d, float delta,
                      double* scratch_d, double* cost_d)
{
    return pm::guarded([&] { pm::huber_cost<float>(stream, count, m, residual_d, delta, scratch_d, cost_d); });
}

int pm_huber_cost_f64(pm_stream_t stream, int64_t count, int64_t m, const double* residual_d, double delta,
                      double* scratch_d, double* cost_d)
{
    return pm::guarded([&] { pm::huber_cost<double>(stream, count, m, residual_d, delta, scratch_d, cost_d); });
}

} // extern "C"
