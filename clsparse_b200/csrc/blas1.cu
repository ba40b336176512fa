// Dense BLAS-1 entry points cldense{S,D,I}* (reference src/library/blas1/*):
// scale, axpy, axpby, add/sub/mul/div, reduce, nrm1, nrm2 and dot.
//
// Every op is one launch. Elementwise ops stream with grid-stride loops sized
// to the SM count. Reductions are one launch as well: each CTA stores a partial
// in the control's scratch area and the last CTA to arrive adds the partials in
// index order (deterministic, no second kernel, no spin-wait), applies the final
// operation (sqrt for nrm2) and writes the device scalar. The reference used two
// launches with a CAS-loop atomic for the second (src/library/blas1/reduce.hpp:102-168,
// src/library/kernels/atomic_reduce.cl:95-113).
//
// Scalars alpha/beta are read from device memory by the kernels, as in the
// reference (src/library/kernels/blas1.cl:59-127). The reference's host-side
// shortcuts for alpha == 0 in scale and axpy (cldense-scale.cpp:41-53,
// cldense-axpy.cpp:50-63, both blocking reads of alpha) are evaluated on the
// device instead, with the same results.
#include <cmath>

#include "device_common.cuh"
#include "internal.h"

namespace clsp {
namespace {

constexpr int kThreads = 256;

enum class Ew : int { Add, Sub, Mul, Div };
enum class Red : int { Plus, Abs, Sqr, Dot };

uint32_t ew_grid(size_t n, int sms) {
    size_t ctas = (n + kThreads * 4 - 1) / (kThreads * 4);
    const size_t cap = static_cast<size_t>(sms) * 16;
    if (ctas > cap) ctas = cap;
    if (ctas == 0) ctas = 1;
    return static_cast<uint32_t>(ctas);
}

uint32_t red_grid(size_t n, int sms) {
    size_t ctas = (n + kThreads * 8 - 1) / (kThreads * 8);
    size_t cap = static_cast<size_t>(sms) * 8;
    if (cap > static_cast<size_t>(kMaxReduceCtas)) cap = kMaxReduceCtas;
    if (ctas > cap) ctas = cap;
    if (ctas == 0) ctas = 1;
    return static_cast<uint32_t>(ctas);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) scale_kernel(size_t n, T* r, const T* __restrict__ y,
                                                         const T* __restrict__ alpha_p) {
    const T a = *alpha_p;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
        r[i] = (a == T(0)) ? T(0) : y[i] * a;
}

// r = y + alpha * x  (alpha == 0: r = y)
template <typename T>
__global__ void __launch_bounds__(kThreads) axpy_kernel(size_t n, T* r, const T* __restrict__ alpha_p,
                                                        const T* x, const T* y) {
    const T a = *alpha_p;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
        r[i] = (a == T(0)) ? y[i] : y[i] + a * x[i];
}

// r = alpha * x + beta * y
template <typename T>
__global__ void __launch_bounds__(kThreads)
    axpby_kernel(size_t n, T* r, const T* __restrict__ alpha_p, const T* x,
                 const T* __restrict__ beta_p, const T* y) {
    const T a = *alpha_p;
    const T b = *beta_p;
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride)
        r[i] = a * x[i] + b * y[i];
}

template <typename T, Ew OP>
__global__ void __launch_bounds__(kThreads) ew_kernel(size_t n, T* r, const T* x, const T* y) {
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const T a = x[i], b = y[i];
        T v;
        if constexpr (OP == Ew::Add) v = a + b;
        if constexpr (OP == Ew::Sub) v = a - b;
        if constexpr (OP == Ew::Mul) v = a * b;
        if constexpr (OP == Ew::Div) v = a / b;
        r[i] = v;
    }
}

// Accumulator type of a reduction: double for floating point, 64-bit integer
// for cldenseIreduce (wraps to 32 bits when stored, as an int sum would).
template <typename T>
struct RedAcc {
    using type = double;
};
template <>
struct RedAcc<int> {
    using type = long long;
};

template <typename T, Red OP>
__global__ void __launch_bounds__(kThreads)
    reduce_kernel(size_t n, const T* __restrict__ x, const T* __restrict__ y, T* out,
                  typename RedAcc<T>::type* partials, uint32_t* ticket) {
    using U = typename RedAcc<T>::type;
    U acc[1] = {U(0)};
    const size_t stride = static_cast<size_t>(gridDim.x) * kThreads;
    for (size_t i = static_cast<size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const U v = static_cast<U>(x[i]);
        if constexpr (OP == Red::Plus) acc[0] += v;
        if constexpr (OP == Red::Abs) acc[0] += v < U(0) ? -v : v;
        if constexpr (OP == Red::Sqr) acc[0] += v * v;
        if constexpr (OP == Red::Dot) acc[0] += v * static_cast<U>(y[i]);
    }
    U tot[1];
    if (dev::grid_reduce_last<1, U>(acc, partials, ticket, tot)) {
        if (threadIdx.x == 0) {
            if constexpr (OP == Red::Sqr) {
                *out = static_cast<T>(sqrt(static_cast<double>(tot[0])));
            } else {
                *out = static_cast<T>(tot[0]);
            }
        }
    }
}

bool sizes_ok(const cldenseVector* a, const cldenseVector* b) {
    return a->num_values == b->num_values;
}

template <typename T>
clsparseStatus do_scale(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* y,
                        clsparseControl c) {
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (!r || !alpha || !y) return clsparseInvalidValue;
    if (!sizes_ok(r, y)) return clsparseInvalidSize;
    const size_t n = r->num_values;
    if (n == 0) return clsparseSuccess;
    DeviceGuard g(c->device);
    scale_kernel<T><<<ew_grid(n, c->sm_count), kThreads, 0, c->stream>>>(
        n, dev_ptr<T>(r->values, r->off_values), dev_ptr<const T>(y->values, y->off_values),
        dev_ptr<const T>(alpha->value, alpha->off_value));
    return finish_call(c);
}

template <typename T>
clsparseStatus do_axpy(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                       const cldenseVector* y, clsparseControl c) {
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (!r || !alpha || !x || !y) return clsparseInvalidValue;
    if (!sizes_ok(r, y) || !sizes_ok(r, x)) return clsparseInvalidSize;
    const size_t n = r->num_values;
    if (n == 0) return clsparseSuccess;
    DeviceGuard g(c->device);
    axpy_kernel<T><<<ew_grid(n, c->sm_count), kThreads, 0, c->stream>>>(
        n, dev_ptr<T>(r->values, r->off_values), dev_ptr<const T>(alpha->value, alpha->off_value),
        dev_ptr<const T>(x->values, x->off_values), dev_ptr<const T>(y->values, y->off_values));
    return finish_call(c);
}

template <typename T>
clsparseStatus do_axpby(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                        const clsparseScalar* beta, const cldenseVector* y, clsparseControl c) {
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (!r || !alpha || !x || !beta || !y) return clsparseInvalidValue;
    if (!sizes_ok(r, y) || !sizes_ok(r, x)) return clsparseInvalidSize;
    const size_t n = r->num_values;
    if (n == 0) return clsparseSuccess;
    DeviceGuard g(c->device);
    axpby_kernel<T><<<ew_grid(n, c->sm_count), kThreads, 0, c->stream>>>(
        n, dev_ptr<T>(r->values, r->off_values), dev_ptr<const T>(alpha->value, alpha->off_value),
        dev_ptr<const T>(x->values, x->off_values), dev_ptr<const T>(beta->value, beta->off_value),
        dev_ptr<const T>(y->values, y->off_values));
    return finish_call(c);
}

template <typename T, Ew OP>
clsparseStatus do_ew(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                     clsparseControl c) {
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (!r || !x || !y) return clsparseInvalidValue;
    if (!sizes_ok(x, y) || !sizes_ok(r, x)) return clsparseInvalidSize;
    const size_t n = x->num_values;
    if (n == 0) return clsparseSuccess;
    DeviceGuard g(c->device);
    ew_kernel<T, OP><<<ew_grid(n, c->sm_count), kThreads, 0, c->stream>>>(
        n, dev_ptr<T>(r->values, r->off_values), dev_ptr<const T>(x->values, x->off_values),
        dev_ptr<const T>(y->values, y->off_values));
    return finish_call(c);
}

template <typename T, Red OP>
clsparseStatus do_reduce(clsparseScalar* s, const cldenseVector* x, const cldenseVector* y,
                         clsparseControl c) {
    using U = typename RedAcc<T>::type;
    clsparseStatus st = check_entry(c);
    if (st != clsparseSuccess) return st;
    if (!s || !x || (OP == Red::Dot && !y)) return clsparseInvalidValue;
    if (OP == Red::Dot && !sizes_ok(x, y)) return clsparseInvalidSize;
    const size_t n = x->num_values;
    DeviceGuard g(c->device);
    U* partials = static_cast<U*>(c->reduce_scratch.ptr);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(static_cast<char*>(c->reduce_scratch.ptr) +
                                                   sizeof(double) * 4 * kMaxReduceCtas);
    const T* yp = (OP == Red::Dot) ? dev_ptr<const T>(y->values, y->off_values) : nullptr;
    reduce_kernel<T, OP><<<red_grid(n, c->sm_count), kThreads, 0, c->stream>>>(
        n, dev_ptr<const T>(x->values, x->off_values), yp, dev_ptr<T>(s->value, s->off_value),
        partials, ticket);
    return finish_call(c);
}

}  // namespace
}  // namespace clsp

using namespace clsp;

extern "C" {

clsparseStatus cldenseSscale(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* y,
                             const clsparseControl control) {
    return do_scale<float>(r, alpha, y, control);
}
clsparseStatus cldenseDscale(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* y,
                             const clsparseControl control) {
    return do_scale<double>(r, alpha, y, control);
}
clsparseStatus cldenseSaxpy(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                            const cldenseVector* y, const clsparseControl control) {
    return do_axpy<float>(r, alpha, x, y, control);
}
clsparseStatus cldenseDaxpy(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                            const cldenseVector* y, const clsparseControl control) {
    return do_axpy<double>(r, alpha, x, y, control);
}
clsparseStatus cldenseSaxpby(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                             const clsparseScalar* beta, const cldenseVector* y,
                             const clsparseControl control) {
    return do_axpby<float>(r, alpha, x, beta, y, control);
}
clsparseStatus cldenseDaxpby(cldenseVector* r, const clsparseScalar* alpha, const cldenseVector* x,
                             const clsparseScalar* beta, const cldenseVector* y,
                             const clsparseControl control) {
    return do_axpby<double>(r, alpha, x, beta, y, control);
}
clsparseStatus cldenseIreduce(clsparseScalar* s, const cldenseVector* x,
                              const clsparseControl control) {
    return do_reduce<int, Red::Plus>(s, x, nullptr, control);
}
clsparseStatus cldenseSreduce(clsparseScalar* s, const cldenseVector* x,
                              const clsparseControl control) {
    return do_reduce<float, Red::Plus>(s, x, nullptr, control);
}
clsparseStatus cldenseDreduce(clsparseScalar* s, const cldenseVector* x,
                              const clsparseControl control) {
    return do_reduce<double, Red::Plus>(s, x, nullptr, control);
}
clsparseStatus cldenseSnrm1(clsparseScalar* s, const cldenseVector* x, const clsparseControl control) {
    return do_reduce<float, Red::Abs>(s, x, nullptr, control);
}
clsparseStatus cldenseDnrm1(clsparseScalar* s, const cldenseVector* x, const clsparseControl control) {
    return do_reduce<double, Red::Abs>(s, x, nullptr, control);
}
clsparseStatus cldenseSnrm2(clsparseScalar* s, const cldenseVector* x, const clsparseControl control) {
    return do_reduce<float, Red::Sqr>(s, x, nullptr, control);
}
clsparseStatus cldenseDnrm2(clsparseScalar* s, const cldenseVector* x, const clsparseControl control) {
    return do_reduce<double, Red::Sqr>(s, x, nullptr, control);
}
clsparseStatus cldenseSdot(clsparseScalar* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_reduce<float, Red::Dot>(r, x, y, control);
}
clsparseStatus cldenseDdot(clsparseScalar* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_reduce<double, Red::Dot>(r, x, y, control);
}
clsparseStatus cldenseSadd(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<float, Ew::Add>(r, x, y, control);
}
clsparseStatus cldenseDadd(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<double, Ew::Add>(r, x, y, control);
}
clsparseStatus cldenseSsub(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<float, Ew::Sub>(r, x, y, control);
}
clsparseStatus cldenseDsub(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<double, Ew::Sub>(r, x, y, control);
}
clsparseStatus cldenseSmul(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<float, Ew::Mul>(r, x, y, control);
}
clsparseStatus cldenseDmul(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<double, Ew::Mul>(r, x, y, control);
}
clsparseStatus cldenseSdiv(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<float, Ew::Div>(r, x, y, control);
}
clsparseStatus cldenseDdiv(cldenseVector* r, const cldenseVector* x, const cldenseVector* y,
                           const clsparseControl control) {
    return do_ew<double, Ew::Div>(r, x, y, control);
}

}  // extern "C"
