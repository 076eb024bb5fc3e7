// simd/simd.h -- host stand-in for the few Apple simd vector types the
// reference's host code (octree.cpp, ANEOS.cpp) uses, so those files compile
// unchanged with g++ into oracle/_ref.  TEST INFRASTRUCTURE ONLY.
// simd_float3 is 16 bytes like Apple's; arithmetic is component-wise float.
// <math.h> brings the float overloads of pow/exp/... into the global
// namespace, as Apple's libc++ headers do.
#ifndef REF_SHIM_SIMD_H
#define REF_SHIM_SIMD_H
#include <math.h>

struct alignas(16) simd_float3 {
    float x, y, z;
    simd_float3() = default;
    simd_float3(float a, float b, float c) : x(a), y(b), z(c) {}
    simd_float3 &operator+=(const simd_float3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    simd_float3 &operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};
struct alignas(8) simd_float2 {
    float x, y;
    simd_float2() = default;
    simd_float2(float a, float b) : x(a), y(b) {}
};
inline simd_float2 operator*(const simd_float2 &a, float s) { return simd_float2(a.x * s, a.y * s); }
inline simd_float2 operator*(float s, const simd_float2 &a) { return simd_float2(s * a.x, s * a.y); }
inline simd_float2 operator+(const simd_float2 &a, const simd_float2 &b) { return simd_float2(a.x + b.x, a.y + b.y); }
struct alignas(16) simd_int3 { int x, y, z; };
struct simd_uint2 { unsigned x, y; };
namespace simd {
typedef simd_float3 float3;
typedef simd_float2 float2;
}
#endif
