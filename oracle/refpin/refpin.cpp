// Test infrastructure (oracle pinning): a C ABI around reference code
// compiled from the reference tree -- BorisPusher (src/Steppers/BorisPusher.h,
// header only), Quaternion (src/Classic/Algorithms/Quaternion.cpp) and
// CoordinateSystemTrafo (src/Classic/Algorithms/CoordinateSystemTrafo.{h,cpp}).
// The tests call these beside the oracle's restatements on the same random
// inputs and require identical doubles.  Nothing in the product links it.
#include "Utility/Inform.h"
#include "Algorithms/CoordinateSystemTrafo.h"
#include "Algorithms/Quaternion.h"
#include "Steppers/BorisPusher.h"

Inform* gmsg = nullptr;

namespace {
Vector_t vec(const double* v) { return Vector_t(v[0], v[1], v[2]); }
void put(const Vector_t& v, double* out) {
    out[0] = v(0);
    out[1] = v(1);
    out[2] = v(2);
}
CoordinateSystemTrafo trafo(const double* origin, const double* quat) {
    return CoordinateSystemTrafo(vec(origin), Quaternion(quat[0], quat[1], quat[2], quat[3]));
}
}  // namespace

extern "C" {

// BorisPusher::kick(R, P, Ef, Bf, dt, mass, charge) (BorisPusher.h:56-113)
void ref_boris_kick(const double* R, double* P, const double* Ef, const double* Bf, double dt, double mass,
                    double charge) {
    BorisPusher pusher;
    Vector_t p = vec(P);
    pusher.kick(vec(R), p, vec(Ef), vec(Bf), dt, mass, charge);
    put(p, P);
}

// BorisPusher::push(R, P, dt) on a position in units of c dt (BorisPusher.h:116-124)
void ref_boris_push_unitless(double* R, const double* P, double dt) {
    BorisPusher pusher;
    Vector_t r = vec(R);
    pusher.push(r, vec(P), dt);
    put(r, R);
}

// getQuaternion(u, ref) (Quaternion.cpp:34-68)
void ref_get_quaternion(const double* u, const double* ref, double* q) {
    Quaternion r = getQuaternion(vec(u), vec(ref));
    for (int i = 0; i < 4; ++i) q[i] = r(i);
}

// Quaternion::getRotationMatrix (Quaternion.cpp:135-150), row major
void ref_rotation_matrix(const double* quat, double* M) {
    Tenzor<double, 3> m = Quaternion(quat[0], quat[1], quat[2], quat[3]).getRotationMatrix();
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[3 * i + j] = m(i, j);
}

// Quaternion::rotate (Quaternion.cpp:120-126)
void ref_quaternion_rotate(const double* quat, const double* v, double* out) {
    put(Quaternion(quat[0], quat[1], quat[2], quat[3]).rotate(vec(v)), out);
}

// CoordinateSystemTrafo(origin, quat).transformTo(r) / rotateTo(r)
void ref_trafo_transform_to(const double* origin, const double* quat, const double* r, double* out) {
    put(trafo(origin, quat).transformTo(vec(r)), out);
}
void ref_trafo_rotate_to(const double* origin, const double* quat, const double* r, double* out) {
    put(trafo(origin, quat).rotateTo(vec(r)), out);
}

// inverted() and left * right: origin (3) and quaternion (4) of the result
void ref_trafo_inverted(const double* origin, const double* quat, double* o_out, double* q_out) {
    CoordinateSystemTrafo t = trafo(origin, quat).inverted();
    put(t.getOrigin(), o_out);
    Quaternion q = t.getRotation();
    for (int i = 0; i < 4; ++i) q_out[i] = q(i);
}
void ref_trafo_compose(const double* lo, const double* lq, const double* ro, const double* rq, double* o_out,
                       double* q_out) {
    CoordinateSystemTrafo t = trafo(lo, lq) * trafo(ro, rq);
    put(t.getOrigin(), o_out);
    Quaternion q = t.getRotation();
    for (int i = 0; i < 4; ++i) q_out[i] = q(i);
}

}  // extern "C"
