// Exact geometric predicates on integer coordinates.
//
// Points are snapped to a power-of-two grid so that every coordinate is an
// integer of at most 41 bits (|x| <= 2^40).  Each predicate is evaluated in
// double precision first with a forward error bound in the style of
// Shewchuk's static filters ("Adaptive Precision Floating-Point Arithmetic
// and Fast Robust Geometric Predicates", 1997); only when the sign is not
// certified does it fall back to exact evaluation in 128-bit and 256-bit
// integer arithmetic.  The same integer coordinates feed both paths, so the
// result is always the exact sign for the snapped points.
//
// Sign conventions (right-handed):
//   orient(a,b,c,d)    = sign det[b-a, c-a, d-a]   (> 0: d above plane abc,
//                        seen with a,b,c counter-clockwise)
//   insphere(a,b,c,d,e) > 0 when e lies strictly inside the circumsphere of
//                        (a,b,c,d) with orient(a,b,c,d) > 0.
#pragma once

#include <cmath>
#include <cstdint>

namespace tg_host {

typedef __int128 i128;
typedef unsigned __int128 u128;

// Signed 256-bit integer, two's complement in four 64-bit limbs.
struct I256 {
    uint64_t w[4];
    static I256 from_i128(i128 v) {
        I256 r;
        const u128 u = (u128)v;
        r.w[0] = (uint64_t)u;
        r.w[1] = (uint64_t)(u >> 64);
        const uint64_t ext = v < 0 ? ~0ull : 0ull;
        r.w[2] = ext;
        r.w[3] = ext;
        return r;
    }
    bool negative() const { return (int64_t)w[3] < 0; }
    bool zero() const { return !(w[0] | w[1] | w[2] | w[3]); }
    int sign() const { return negative() ? -1 : (zero() ? 0 : 1); }
    I256 operator+(const I256& o) const {
        I256 r;
        u128 carry = 0;
        for (int i = 0; i < 4; i++) {
            const u128 s = (u128)w[i] + o.w[i] + carry;
            r.w[i] = (uint64_t)s;
            carry = s >> 64;
        }
        return r;
    }
    I256 neg() const {
        I256 r;
        u128 carry = 1;
        for (int i = 0; i < 4; i++) {
            const u128 s = (u128)(~w[i]) + carry;
            r.w[i] = (uint64_t)s;
            carry = s >> 64;
        }
        return r;
    }
    I256 operator-(const I256& o) const { return *this + o.neg(); }
};

// Exact product of two signed 128-bit integers (|a|,|b| < 2^127).
inline I256 mul_i128(i128 a, i128 b) {
    const bool neg = (a < 0) != (b < 0);
    const u128 ua = a < 0 ? (u128)(-a) : (u128)a;
    const u128 ub = b < 0 ? (u128)(-b) : (u128)b;
    const uint64_t a0 = (uint64_t)ua, a1 = (uint64_t)(ua >> 64);
    const uint64_t b0 = (uint64_t)ub, b1 = (uint64_t)(ub >> 64);
    const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
    I256 r;
    r.w[0] = (uint64_t)p00;
    u128 mid = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
    r.w[1] = (uint64_t)mid;
    u128 hi = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + (uint64_t)p11;
    r.w[2] = (uint64_t)hi;
    r.w[3] = (uint64_t)((hi >> 64) + (p11 >> 64));
    return neg ? r.neg() : r;
}

struct IPoint { int64_t x, y, z; };

// 3x3 determinant of integer row vectors with entries below 2^42 in
// magnitude: every term stays below 2^126.
inline i128 det3_exact(int64_t ax, int64_t ay, int64_t az, int64_t bx, int64_t by, int64_t bz,
                       int64_t cx, int64_t cy, int64_t cz) {
    const i128 m0 = (i128)by * cz - (i128)bz * cy;
    const i128 m1 = (i128)bx * cz - (i128)bz * cx;
    const i128 m2 = (i128)bx * cy - (i128)by * cx;
    return (i128)ax * m0 - (i128)ay * m1 + (i128)az * m2;
}

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53

inline int orient(const IPoint& a, const IPoint& b, const IPoint& c, const IPoint& d) {
    const double ux = (double)(b.x - a.x), uy = (double)(b.y - a.y), uz = (double)(b.z - a.z);
    const double vx = (double)(c.x - a.x), vy = (double)(c.y - a.y), vz = (double)(c.z - a.z);
    const double wx = (double)(d.x - a.x), wy = (double)(d.y - a.y), wz = (double)(d.z - a.z);
    const double m0 = vy * wz - vz * wy, m1 = vx * wz - vz * wx, m2 = vx * wy - vy * wx;
    const double det = ux * m0 - uy * m1 + uz * m2;
    const double perm = std::fabs(ux) * (std::fabs(vy * wz) + std::fabs(vz * wy)) +
                        std::fabs(uy) * (std::fabs(vx * wz) + std::fabs(vz * wx)) +
                        std::fabs(uz) * (std::fabs(vx * wy) + std::fabs(vy * wx));
    const double bound = 16.0 * kEps * perm;
    if (det > bound) return 1;
    if (det < -bound) return -1;
    const i128 e = det3_exact(b.x - a.x, b.y - a.y, b.z - a.z, c.x - a.x, c.y - a.y, c.z - a.z,
                              d.x - a.x, d.y - a.y, d.z - a.z);
    return e > 0 ? 1 : (e < 0 ? -1 : 0);
}

inline int insphere(const IPoint& a, const IPoint& b, const IPoint& c, const IPoint& d, const IPoint& e) {
    const double ax = (double)(a.x - e.x), ay = (double)(a.y - e.y), az = (double)(a.z - e.z);
    const double bx = (double)(b.x - e.x), by = (double)(b.y - e.y), bz = (double)(b.z - e.z);
    const double cx = (double)(c.x - e.x), cy = (double)(c.y - e.y), cz = (double)(c.z - e.z);
    const double dx = (double)(d.x - e.x), dy = (double)(d.y - e.y), dz = (double)(d.z - e.z);
    const double la = ax * ax + ay * ay + az * az, lb = bx * bx + by * by + bz * bz;
    const double lc = cx * cx + cy * cy + cz * cz, ld = dx * dx + dy * dy + dz * dz;
    auto d3 = [](double px, double py, double pz, double qx, double qy, double qz, double rx, double ry, double rz, double* perm) {
        *perm = std::fabs(px) * (std::fabs(qy * rz) + std::fabs(qz * ry)) +
                std::fabs(py) * (std::fabs(qx * rz) + std::fabs(qz * rx)) +
                std::fabs(pz) * (std::fabs(qx * ry) + std::fabs(qy * rx));
        return px * (qy * rz - qz * ry) - py * (qx * rz - qz * rx) + pz * (qx * ry - qy * rx);
    };
    double pA, pB, pC, pD;
    const double dBCD = d3(bx, by, bz, cx, cy, cz, dx, dy, dz, &pA);
    const double dACD = d3(ax, ay, az, cx, cy, cz, dx, dy, dz, &pB);
    const double dABD = d3(ax, ay, az, bx, by, bz, dx, dy, dz, &pC);
    const double dABC = d3(ax, ay, az, bx, by, bz, cx, cy, cz, &pD);
    // det of rows (p - e, |p - e|^2); e inside <=> det < 0 for orient(a,b,c,d) > 0
    const double det = -la * dBCD + lb * dACD - lc * dABD + ld * dABC;
    const double perm = la * pA + lb * pB + lc * pC + ld * pD;
    const double bound = 32.0 * kEps * perm;
    if (det > bound) return -1;
    if (det < -bound) return 1;
    const int64_t Ax = a.x - e.x, Ay = a.y - e.y, Az = a.z - e.z;
    const int64_t Bx = b.x - e.x, By = b.y - e.y, Bz = b.z - e.z;
    const int64_t Cx = c.x - e.x, Cy = c.y - e.y, Cz = c.z - e.z;
    const int64_t Dx = d.x - e.x, Dy = d.y - e.y, Dz = d.z - e.z;
    const i128 LA = (i128)Ax * Ax + (i128)Ay * Ay + (i128)Az * Az;
    const i128 LB = (i128)Bx * Bx + (i128)By * By + (i128)Bz * Bz;
    const i128 LC = (i128)Cx * Cx + (i128)Cy * Cy + (i128)Cz * Cz;
    const i128 LD = (i128)Dx * Dx + (i128)Dy * Dy + (i128)Dz * Dz;
    const I256 t0 = mul_i128(LA, det3_exact(Bx, By, Bz, Cx, Cy, Cz, Dx, Dy, Dz));
    const I256 t1 = mul_i128(LB, det3_exact(Ax, Ay, Az, Cx, Cy, Cz, Dx, Dy, Dz));
    const I256 t2 = mul_i128(LC, det3_exact(Ax, Ay, Az, Bx, By, Bz, Dx, Dy, Dz));
    const I256 t3 = mul_i128(LD, det3_exact(Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz));
    const I256 sum = (t1 - t0) - t2 + t3;
    return -sum.sign();
}

}  // namespace tg_host
