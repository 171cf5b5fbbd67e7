// Minimal column-major matrix/vector/quaternion types with the names the
// reference's headers use (matrix.h, material.h), so that those headers
// compile as host C++ for the CPU checker.  Only the operations the compiled
// files name are provided; the checker feeds its own matrices and never
// relies on these for numerics.
#pragma once
#include <cmath>

namespace glm {

struct vec2 { float x = 0, y = 0; vec2() = default; vec2(float a, float b) : x(a), y(b) {} };
struct vec3 {
    float x = 0, y = 0, z = 0;
    vec3() = default;
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return i == 0 ? x : i == 1 ? y : z; }
    float operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
};
struct vec4 {
    float x = 0, y = 0, z = 0, w = 0;
    vec4() = default;
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    float& operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    float operator[](int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};

struct mat4 {
    vec4 c[4];
    mat4() { for (int i = 0; i < 4; ++i) c[i][i] = 1.f; }
    mat4(float a0, float a1, float a2, float a3, float b0, float b1, float b2, float b3,
         float c0, float c1, float c2, float c3, float d0, float d1, float d2, float d3) {
        c[0] = vec4(a0, a1, a2, a3); c[1] = vec4(b0, b1, b2, b3);
        c[2] = vec4(c0, c1, c2, c3); c[3] = vec4(d0, d1, d2, d3);
    }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};

struct mat3 {
    vec3 c[3];
    mat3() { for (int i = 0; i < 3; ++i) c[i][i] = 1.f; }
    explicit mat3(const mat4& m) { for (int i = 0; i < 3; ++i) c[i] = vec3(m[i].x, m[i].y, m[i].z); }
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};

inline mat3 operator*(const mat3& a, const mat3& b) {
    mat3 r;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            r[j][i] = a[0][i] * b[j][0] + a[1][i] * b[j][1] + a[2][i] * b[j][2];
    return r;
}

inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r;
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i)
            r[j][i] = a[0][i] * b[j][0] + a[1][i] * b[j][1] + a[2][i] * b[j][2] + a[3][i] * b[j][3];
    return r;
}

inline mat3 inverse(const mat3& m) {
    float a = m[0][0], b = m[1][0], c = m[2][0];
    float d = m[0][1], e = m[1][1], f = m[2][1];
    float g = m[0][2], h = m[1][2], k = m[2][2];
    float A = e * k - f * h, B = -(d * k - f * g), C = d * h - e * g;
    float det = a * A + b * B + c * C;
    float id = 1.f / det;
    mat3 r;
    r[0][0] = A * id; r[1][0] = -(b * k - c * h) * id; r[2][0] = (b * f - c * e) * id;
    r[0][1] = B * id; r[1][1] = (a * k - c * g) * id;  r[2][1] = -(a * f - c * d) * id;
    r[0][2] = C * id; r[1][2] = -(a * h - b * g) * id; r[2][2] = (a * e - b * d) * id;
    return r;
}

struct quat {
    float w = 1, x = 0, y = 0, z = 0;
    quat() = default;
    quat(float W, float X, float Y, float Z) : w(W), x(X), y(Y), z(Z) {}
    float& operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};

}  // namespace glm
