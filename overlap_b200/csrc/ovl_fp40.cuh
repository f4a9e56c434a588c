// 40-bit storage of the mode fields (precision OVL_PREC_FP40): each real is
// the FP64 value rounded to its top 40 bits -- sign, 11-bit exponent and 28
// mantissa bits, relative rounding at most 2^-29 -- kept as the upper 32-bit
// word of the double in the field and the next 8 bits in an extension byte
// array.  Decoding is a register move (the bits are the double's own), so a
// kernel computing in FP64 pays no conversion instructions.  Per complex
// number: uint2 (8 bytes) in the field + 2 extension bytes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ovl_device.cuh"

namespace ovl {

__device__ __forceinline__ double dec40(unsigned h, unsigned char l) {
    return __hiloint2double((int)h, (int)((unsigned)l << 24));
}

// Round to nearest on the 40-bit boundary (adding half a unit of the last
// kept bit to the magnitude bits carries into the exponent when needed).
__device__ __forceinline__ void enc40(double x, unsigned &h, unsigned char &l) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x) + (1ull << 23);
    h = (unsigned)(b >> 32);
    l = (unsigned char)((b >> 24) & 0xffu);
}

// The extension bytes of one site and mode block sit together: for each
// (block, site, lane) 16 bytes -- re, im of the 8 spinor components -- so a
// warp reads the extensions of a site in one 512-byte request.  Byte offset of
// the (re, im) pair of complex element i of the mode-block layout
// ((block * V + site) * 8 + component) * 32 + lane:
__host__ __device__ __forceinline__ size_t lo_byte(size_t i) {
    return (((i >> 8) << 5) + (i & 31)) * 16 + 2 * ((i >> 5) & 7);
}

// Read-only views of a mode field that hand out complex doubles.
template <typename T> struct SrcPlain {
    const cpx<T> *p;
    __device__ __forceinline__ cpx<double> operator()(size_t i) const {
        const cpx<T> v = ld(p + i);
        return mk<double>((double)v.re, (double)v.im);
    }
};
struct Src40 {
    const uint2 *hi;
    const unsigned char *lo;
    __device__ __forceinline__ cpx<double> operator()(size_t i) const {
        const uint2 h = __ldg(hi + i);
        const uchar2 l = __ldg(reinterpret_cast<const uchar2 *>(lo + lo_byte(i)));
        return mk<double>(dec40(h.x, l.x), dec40(h.y, l.y));
    }
};

__device__ __forceinline__ void store40(uint2 *hi, unsigned char *lo, size_t i, double re, double im) {
    unsigned hx, hy;
    unsigned char lx, ly;
    enc40(re, hx, lx);
    enc40(im, hy, ly);
    hi[i] = make_uint2(hx, hy);
    *reinterpret_cast<uchar2 *>(lo + lo_byte(i)) = make_uchar2(lx, ly);
}

}  // namespace ovl
