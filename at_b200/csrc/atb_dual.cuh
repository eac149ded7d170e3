/*
 * Forward-mode dual numbers for the tangent kernel: a value and K partial
 * derivatives, with the arithmetic the integrators use (+, -, *, /, sin, tan,
 * cos, exp).  The pass-method templates in atb_physics.cuh and
 * track_kernel.cuh run unchanged on this type, which propagates the Jacobian
 * of every operation exactly (no finite differences).  Values are computed
 * with the plain operators (the tangent unit is compiled without FMA
 * contraction, so they equal the exact tracking kernel's); the derivative
 * updates use explicit fma(), which that flag does not touch.
 */
#ifndef ATB_DUAL_CUH
#define ATB_DUAL_CUH

namespace atb {

/* the double overloads stay visible next to the dual ones below */
using ::sin;
using ::cos;
using ::tan;
using ::exp;

template <int K>
struct Dual {
    double v;
    double d[K];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < K; ++i) d[i] = 0.0;
    }
    __device__ __forceinline__ Dual& operator+=(const Dual& o) { return *this = *this + o; }
    __device__ __forceinline__ Dual& operator-=(const Dual& o) { return *this = *this - o; }
    __device__ __forceinline__ Dual& operator*=(const Dual& o) { return *this = *this * o; }
    __device__ __forceinline__ Dual& operator/=(const Dual& o) { return *this = *this / o; }
    __device__ __forceinline__ Dual& operator+=(double o) { v += o; return *this; }
    __device__ __forceinline__ Dual& operator-=(double o) { v -= o; return *this; }
    __device__ __forceinline__ Dual& operator*=(double o) { return *this = *this * o; }
    __device__ __forceinline__ Dual& operator/=(double o) { return *this = *this / o; }

    friend __device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v + b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i];
        return r;
    }
    friend __device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v - b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i];
        return r;
    }
    friend __device__ __forceinline__ Dual operator-(const Dual& a) {
        Dual r;
        r.v = -a.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
        return r;
    }
    friend __device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v * b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = fma(a.d[i], b.v, a.v * b.d[i]);
        return r;
    }
    friend __device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v / b.v;
        const double ib = 1.0 / b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = fma(-r.v, b.d[i], a.d[i]) * ib;
        return r;
    }
    /* mixed forms keep a constant operand from carrying zero derivatives */
    friend __device__ __forceinline__ Dual operator+(const Dual& a, double b) {
        Dual r = a;
        r.v = a.v + b;
        return r;
    }
    friend __device__ __forceinline__ Dual operator+(double a, const Dual& b) { return b + a; }
    friend __device__ __forceinline__ Dual operator-(const Dual& a, double b) {
        Dual r = a;
        r.v = a.v - b;
        return r;
    }
    friend __device__ __forceinline__ Dual operator-(double a, const Dual& b) {
        Dual r;
        r.v = a - b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = -b.d[i];
        return r;
    }
    friend __device__ __forceinline__ Dual operator*(const Dual& a, double b) {
        Dual r;
        r.v = a.v * b;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b;
        return r;
    }
    friend __device__ __forceinline__ Dual operator*(double a, const Dual& b) { return b * a; }
    friend __device__ __forceinline__ Dual operator/(const Dual& a, double b) {
        Dual r;
        r.v = a.v / b;
        const double ib = 1.0 / b;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * ib;
        return r;
    }
    friend __device__ __forceinline__ Dual operator/(double a, const Dual& b) {
        Dual r;
        r.v = a / b.v;
        const double s = -r.v / b.v;
#pragma unroll
        for (int i = 0; i < K; ++i) r.d[i] = s * b.d[i];
        return r;
    }
};

/* acc + a*b and acc - a*b: the value rounded as the plain expression (the
 * product, then the sum), each derivative slot in two FMAs instead of a
 * product, an FMA and an add.  The double forms are the plain expressions, so
 * the tracking kernels compute what they computed before. */
__device__ __forceinline__ double madd(double acc, double a, double b) { return acc + a * b; }
__device__ __forceinline__ double msub(double acc, double a, double b) { return acc - a * b; }

template <int K>
__device__ __forceinline__ Dual<K> madd(const Dual<K>& acc, const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = acc.v + a.v * b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = fma(a.d[i], b.v, fma(a.v, b.d[i], acc.d[i]));
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> madd(const Dual<K>& acc, double a, const Dual<K>& b) {
    Dual<K> r;
    r.v = acc.v + a * b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = fma(a, b.d[i], acc.d[i]);
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> msub(const Dual<K>& acc, double a, const Dual<K>& b) {
    Dual<K> r;
    r.v = acc.v - a * b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = fma(-a, b.d[i], acc.d[i]);
    return r;
}

/* One complex Horner step on dual numbers, (re, im) <- (re, im)(x + i y) +
 * (b + i a), values in the reference's order (re x - im y + b,
 * im x + re y + a) and each derivative slot of a component in four fused
 * operations instead of five. */
template <int K>
__device__ __forceinline__ void horner_step_dual(Dual<K>& re, Dual<K>& im, const Dual<K>& x,
                                                 const Dual<K>& y, double b, double a) {
    Dual<K> nr, ni;
    nr.v = re.v * x.v - im.v * y.v + b;
    ni.v = im.v * x.v + re.v * y.v + a;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        nr.d[i] = fma(re.d[i], x.v, fma(re.v, x.d[i], fma(-im.d[i], y.v, -(im.v * y.d[i]))));
        ni.d[i] = fma(im.d[i], x.v, fma(im.v, x.d[i], fma(re.d[i], y.v, re.v * y.d[i])));
    }
    re = nr;
    im = ni;
}

/* sin and cos are called separately (not sincos) so the value is exactly
 * the one the double kernels compute */
template <int K>
__device__ __forceinline__ Dual<K> sin(const Dual<K>& a) {
    Dual<K> r;
    const double s = ::sin(a.v), c = ::cos(a.v);
    r.v = s;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = c * a.d[i];
    return r;
}

template <int K>
__device__ __forceinline__ Dual<K> cos(const Dual<K>& a) {
    Dual<K> r;
    const double s = ::sin(a.v), c = ::cos(a.v);
    r.v = c;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = -s * a.d[i];
    return r;
}

template <int K>
__device__ __forceinline__ Dual<K> tan(const Dual<K>& a) {
    Dual<K> r;
    r.v = ::tan(a.v);
    const double s = 1.0 + r.v * r.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = s * a.d[i];
    return r;
}

template <int K>
__device__ __forceinline__ Dual<K> exp(const Dual<K>& a) {
    Dual<K> r;
    r.v = ::exp(a.v);
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = r.v * a.d[i];
    return r;
}

/* the value of a scalar (for comparisons and loss tests) */
__device__ __forceinline__ double val(double x) { return x; }
template <int K>
__device__ __forceinline__ double val(const Dual<K>& x) { return x.v; }

template <class T>
struct is_dual { static constexpr bool value = false; };
template <int K>
struct is_dual<Dual<K>> { static constexpr bool value = true; };

}  // namespace atb

#endif  // ATB_DUAL_CUH
