// Host-only stand-in for the half type and the load intrinsic the physics
// headers name; the algebra check never touches half values.
#pragma once
struct __half { unsigned short x; };
template <class T> inline T __ldg(const T* p) { return *p; }
inline float __half2float(__half) { return 0.f; }
inline __half __float2half(float) { return __half{}; }
inline __half __double2half(double) { return __half{}; }
inline __half __float2half_rn(float) { return __half{}; }
