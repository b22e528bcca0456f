/*
 * Minimal stand-in for OpenMM's Vec3, written for the oracle harness only.  OpenMM is not
 * installed in this environment; this header provides the small part of its interface that
 * the reference's Reference-platform kernel uses (component access, +, -, scaling, dot).
 */
#ifndef SHIM_OPENMM_VEC3_H_
#define SHIM_OPENMM_VEC3_H_
namespace OpenMM {
class Vec3 {
public:
    Vec3() { d[0] = d[1] = d[2] = 0.0; }
    Vec3(double x, double y, double z) { d[0] = x; d[1] = y; d[2] = z; }
    double operator[](int i) const { return d[i]; }
    double& operator[](int i) { return d[i]; }
    Vec3 operator+(const Vec3& o) const { return Vec3(d[0]+o.d[0], d[1]+o.d[1], d[2]+o.d[2]); }
    Vec3 operator-(const Vec3& o) const { return Vec3(d[0]-o.d[0], d[1]-o.d[1], d[2]-o.d[2]); }
    Vec3 operator-() const { return Vec3(-d[0], -d[1], -d[2]); }
    Vec3 operator*(double s) const { return Vec3(d[0]*s, d[1]*s, d[2]*s); }
    Vec3& operator+=(const Vec3& o) { d[0] += o.d[0]; d[1] += o.d[1]; d[2] += o.d[2]; return *this; }
    Vec3& operator-=(const Vec3& o) { d[0] -= o.d[0]; d[1] -= o.d[1]; d[2] -= o.d[2]; return *this; }
    Vec3& operator*=(double s) { d[0] *= s; d[1] *= s; d[2] *= s; return *this; }
    bool operator==(const Vec3& o) const { return d[0] == o.d[0] && d[1] == o.d[1] && d[2] == o.d[2]; }
    bool operator!=(const Vec3& o) const { return !(*this == o); }
    double dot(const Vec3& o) const { return d[0]*o.d[0] + d[1]*o.d[1] + d[2]*o.d[2]; }
private:
    double d[3];
};
}
#endif
