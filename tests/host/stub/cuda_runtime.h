// Host-only stand-in so the device physics headers compile with g++ (tests):
// the float2 type and the packed FP32 intrinsics (each half one IEEE fused
// multiply-add, addition or multiplication, as the device instructions).
#pragma once
#include <cmath>
struct float2 {
    float x, y;
};
inline float2 make_float2(float a, float b) { return float2{a, b}; }
inline float2 __ffma2_rn(float2 a, float2 b, float2 c) { return {std::fmaf(a.x, b.x, c.x), std::fmaf(a.y, b.y, c.y)}; }
inline float2 __fadd2_rn(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
inline float2 __fmul2_rn(float2 a, float2 b) { return {a.x * b.x, a.y * b.y}; }
