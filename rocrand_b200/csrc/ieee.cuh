// ieee.cuh -- single IEEE operations with round-to-nearest (or truncation where named), the
// same on the device and on the host.
//
// The distribution functors (dist.cuh) spell every rounding step, because their outputs must
// equal the reference's host generators bit for bit: on the device each operation is the
// matching _rn intrinsic, which the compiler never contracts into an FMA; on the host it is
// the plain C++ operation, and every host file of the library is compiled with
// -ffp-contract=off, so it is rounded once, as written.  The host forms let the CPU path of
// the host generators (cpu_generators.cpp) run the very functors the kernels run.
#pragma once

#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define RB_HD __host__ __device__ __forceinline__
#else
#define RB_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define RB_PICK(device_form, host_form) return device_form
#else
#define RB_PICK(device_form, host_form) return host_form
#endif

namespace rb200
{
namespace ieee
{

RB_HD float fadd(float a, float b) { RB_PICK(__fadd_rn(a, b), a + b); }
RB_HD float fsub(float a, float b) { RB_PICK(__fsub_rn(a, b), a - b); }
RB_HD float fmul(float a, float b) { RB_PICK(__fmul_rn(a, b), a * b); }
RB_HD float ffma(float a, float b, float c) { RB_PICK(__fmaf_rn(a, b, c), std::fma(a, b, c)); }
RB_HD float fsqrt(float a) { RB_PICK(__fsqrt_rn(a), std::sqrt(a)); }
RB_HD double dadd(double a, double b) { RB_PICK(__dadd_rn(a, b), a + b); }
RB_HD double dsub(double a, double b) { RB_PICK(__dsub_rn(a, b), a - b); }
RB_HD double dmul(double a, double b) { RB_PICK(__dmul_rn(a, b), a * b); }
RB_HD double dfma(double a, double b, double c) { RB_PICK(__fma_rn(a, b, c), std::fma(a, b, c)); }
RB_HD double dsqrt(double a) { RB_PICK(__dsqrt_rn(a), std::sqrt(a)); }
RB_HD float u2f(uint32_t v) { RB_PICK(__uint2float_rn(v), static_cast<float>(v)); }
RB_HD double u2d(uint32_t v) { RB_PICK(__uint2double_rn(v), static_cast<double>(v)); }
RB_HD double ull2d(unsigned long long v) { RB_PICK(__ull2double_rn(v), static_cast<double>(v)); }
RB_HD uint32_t d2u_rz(double v) { RB_PICK(__double2uint_rz(v), static_cast<uint32_t>(v)); }
RB_HD float d2f(double v) { RB_PICK(__double2float_rn(v), static_cast<float>(v)); }

// The transcendental functions of the fp32 transforms: the device's own library functions
// on the device (within an ulp or two of the host's), the C library's on the host (the
// functions the reference's host generators call, so the host path is bit-exact).
RB_HD float logf_(float x) { RB_PICK(logf(x), std::log(x)); }
RB_HD float expf_(float x) { RB_PICK(expf(x), std::exp(x)); }
RB_HD double exp_(double x) { RB_PICK(exp(x), std::exp(x)); }
RB_HD void sincosf_(float x, float* s, float* c)
{
#if defined(__CUDA_ARCH__)
    sincosf(x, s, c);
#else
    *s = std::sin(x);
    *c = std::cos(x);
#endif
}

} // namespace ieee
} // namespace rb200
