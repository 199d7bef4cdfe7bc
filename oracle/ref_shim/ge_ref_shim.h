/*
 * ge_ref_shim.h -- minimal stand-ins for the vendor headers that the
 * reference's precompiled header (GalaxyEngine/include/pch.h) would provide,
 * just enough to compile the reference's Physics/morton.cpp and
 * Physics/quadtree.cpp unmodified for the oracle pin (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY.  glm (1.0.1, cmake/glm.cmake) and raylib are
 * not present in this image; those two sources use glm vectors only through
 * component-wise + - * / and constructors, and raylib only for the Color
 * type, which is all this file defines.  Each operator below performs the
 * plain IEEE float operation per component, which is what glm's own
 * component-wise operators compute.
 */
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <limits>
#include <numeric>
#include <vector>

struct Color { unsigned char r, g, b, a; };

namespace glm {

struct vec2 {
    float x, y;
    vec2() : x(0.0f), y(0.0f) {}
    vec2(float a, float b) : x(a), y(b) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2 &operator+=(const vec2 &o) { x += o.x; y += o.y; return *this; }
    vec2 &operator-=(const vec2 &o) { x -= o.x; y -= o.y; return *this; }
    vec2 &operator*=(float s) { x *= s; y *= s; return *this; }
    vec2 &operator/=(float s) { x /= s; y /= s; return *this; }
};
inline vec2 operator+(vec2 a, vec2 b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(vec2 a, vec2 b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator+(vec2 a, float s) { return vec2(a.x + s, a.y + s); }
inline vec2 operator-(vec2 a, float s) { return vec2(a.x - s, a.y - s); }
inline vec2 operator*(vec2 a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator*(float s, vec2 a) { return vec2(s * a.x, s * a.y); }
inline vec2 operator/(vec2 a, float s) { return vec2(a.x / s, a.y / s); }

struct vec3 {
    float x, y, z;
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3 &operator+=(const vec3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    vec3 &operator-=(const vec3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    vec3 &operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    vec3 &operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};
inline vec3 operator+(vec3 a, vec3 b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(vec3 a, vec3 b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator+(vec3 a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(vec3 a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator*(vec3 a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, vec3 a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(vec3 a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }

struct vec4 {
    float x, y, z, w;
    vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

}  // namespace glm
