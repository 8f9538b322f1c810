// softening.cuh — spline-softened gravity kernels shared by the FP64 and the
// mixed-precision gravity walks.
#pragma once

namespace sphgpu {

// Hernquist & Katz (1989) potential / force kernels (src/bhtree.cpp:318-345)
template <typename T>
__device__ __forceinline__ T hk_f(T r, T h)
{
    const T e = h * T(0.5);
    const T u = r / e;
    if(u < T(1.0)) return (T(-0.5) * u * u * (T(1.0 / 3.0) - T(3.0 / 20) * u * u + u * u * u / T(20)) + T(1.4)) / e;
    if(u < T(2.0))
        return T(-1.0) / (T(15) * r) + (-u * u * (T(4.0 / 3.0) - u + T(0.3) * u * u - u * u * u / T(30)) + T(1.6)) / e;
    return T(1) / r;
}

template <typename T>
__device__ __forceinline__ T hk_g(T r, T h)
{
    const T e = h * T(0.5);
    const T u = r / e;
    if(u < T(1.0)) return (T(4.0 / 3.0) - T(1.2) * u * u + T(0.5) * u * u * u) / (e * e * e);
    if(u < T(2.0))
        return (T(-1.0 / 15) + T(8.0 / 3) * u * u * u - T(3) * u * u * u * u + T(1.2) * u * u * u * u * u
                - u * u * u * u * u * u / T(6.0))
            / (r * r * r);
    return T(1) / (r * r * r);
}

}  // namespace sphgpu
