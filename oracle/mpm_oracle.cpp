// ORACLE / TEST INFRASTRUCTURE ONLY.  Loaded by tests/, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py as the checker; never by the product path.
//
// Scalar restatement of CRESSim-MPM's substep algorithms, written from the reference's code
// (citations are `file:line` inside the reference project), templated on the scalar type:
//   T = float   follows the reference's single-precision operation order one to one, so on the
//               same inputs it reproduces the reference's CPU solver; it is pinned against the
//               reference's own headers (oracle/ref_driver.cpp) by tests/test_oracle_pin.py.
//   T = double  the FP64 oracle used for tolerance checks of the float kernels.
// The only deliberate difference from the reference is the 3x3 SVD (mpm_oracle_svd.h).
//
// Parity-relevant reference behaviours kept on purpose (see the reference lines cited):
//   - eCoRotational falls through to linear (StVK) elasticity (constitutive_models.h:109-113)
//   - grid mass cutoffs 1e-4 (MLS, standard) and 1e-8 (PB) keep momentum in light nodes
//   - the APIC matrix is 4/dx * sum w d v^T stored as M(r,c) = d_r v_c (vec3 outerProduct is
//     b a^T, mat33.h:287-306; mls_mpm_algorithm.h:361)
//   - standard-MPM weight gradients are in grid units (shape_functions.h:62-75)
//   - trilinear SDF weights index x as the low bit while values index z (sdf.h:243-276)
//   - slicer normals in G2P stay in the shape's local frame (mpm_rigid_contact.h:466-471)
//   - PB-MPM's rotation target is the transpose of the polar rotation of targetF (svd3.h:1271-1274)

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "crmpm_b200.h"
#include "mpm_oracle_svd.h"

namespace orc
{
    template <typename T>
    struct V3
    {
        T x = 0, y = 0, z = 0;
        V3() = default;
        V3(T a, T b, T c) : x(a), y(b), z(c) {}
        V3 operator+(const V3 &o) const { return V3(x + o.x, y + o.y, z + o.z); }
        V3 operator-(const V3 &o) const { return V3(x - o.x, y - o.y, z - o.z); }
        V3 operator*(T s) const { return V3(x * s, y * s, z * s); }
        V3 operator/(T s) const { return V3(x / s, y / s, z / s); }
        V3 mul(const V3 &o) const { return V3(x * o.x, y * o.y, z * o.z); }
        V3 div(const V3 &o) const { return V3(x / o.x, y / o.y, z / o.z); }
        T dot(const V3 &o) const { return x * o.x + y * o.y + z * o.z; }
        V3 cross(const V3 &o) const { return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
        T sq() const { return x * x + y * y + z * z; }
        T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
        T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    };

    // Column-major 3x3 (the reference's Mat3x3f is three columns, mat33.h:46-53).
    template <typename T>
    struct M3
    {
        V3<T> c0, c1, c2;
        static M3 I() { M3 m; m.c0.x = 1; m.c1.y = 1; m.c2.z = 1; return m; }
        T operator()(int r, int c) const { return (c == 0 ? c0 : (c == 1 ? c1 : c2))[r]; }
        T &at(int r, int c) { return (c == 0 ? c0 : (c == 1 ? c1 : c2))[r]; }
        // mat33.h:123-126: ((col0 * v.x) + (col1 * v.y)) + (col2 * v.z)
        V3<T> operator*(const V3<T> &v) const { return c0 * v.x + c1 * v.y + c2 * v.z; }
        M3 operator*(const M3 &o) const { M3 r; r.c0 = (*this) * o.c0; r.c1 = (*this) * o.c1; r.c2 = (*this) * o.c2; return r; }
        M3 operator*(T s) const { M3 r; r.c0 = c0 * s; r.c1 = c1 * s; r.c2 = c2 * s; return r; }
        M3 operator+(const M3 &o) const { M3 r; r.c0 = c0 + o.c0; r.c1 = c1 + o.c1; r.c2 = c2 + o.c2; return r; }
        M3 operator-(const M3 &o) const { M3 r; r.c0 = c0 - o.c0; r.c1 = c1 - o.c1; r.c2 = c2 - o.c2; return r; }
        // mat33.h:219-232
        T det() const
        {
            T a = (*this)(0, 0), b = (*this)(0, 1), c = (*this)(0, 2);
            T d = (*this)(1, 0), e = (*this)(1, 1), f = (*this)(1, 2);
            T g = (*this)(2, 0), h = (*this)(2, 1), i = (*this)(2, 2);
            return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
        }
        M3 T_() const
        {
            M3 r;
            r.c0 = V3<T>(c0.x, c1.x, c2.x);
            r.c1 = V3<T>(c0.y, c1.y, c2.y);
            r.c2 = V3<T>(c0.z, c1.z, c2.z);
            return r;
        }
        T trace() const { return c0.x + c1.y + c2.z; }
        // mat33.h:256-283
        M3 inverse() const
        {
            T a = (*this)(0, 0), b = (*this)(0, 1), c = (*this)(0, 2);
            T d = (*this)(1, 0), e = (*this)(1, 1), f = (*this)(1, 2);
            T g = (*this)(2, 0), h = (*this)(2, 1), i = (*this)(2, 2);
            T dt = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
            if (std::fabs(dt) < T(1e-6f))
                return M3();
            T inv = T(1) / dt;
            M3 adj;
            adj.c0 = V3<T>((e * i - f * h), -(b * i - c * h), (b * f - c * e));
            adj.c1 = V3<T>(-(d * i - f * g), (a * i - c * g), -(a * f - c * d));
            adj.c2 = V3<T>((d * h - e * g), -(a * h - b * g), (a * e - b * d));
            return adj * inv;
        }
        // this = other * this (mat33.h:208-214)
        void leftMul(const M3 &o) { c0 = o * c0; c1 = o * c1; c2 = o * c2; }
    };

    // Vec3 outerProduct as defined by the reference: result(r, c) = a_c * b_r (mat33.h:287-306).
    template <typename T>
    M3<T> refOuter(const V3<T> &a, const V3<T> &b)
    {
        M3<T> m;
        m.c0 = V3<T>(a.x * b.x, a.x * b.y, a.x * b.z);
        m.c1 = V3<T>(a.y * b.x, a.y * b.y, a.y * b.z);
        m.c2 = V3<T>(a.z * b.x, a.z * b.y, a.z * b.z);
        return m;
    }

    template <typename T> T rsqrtT(T v) { return T(1) / std::sqrt(v); } // host rsqrtf, cuda_compat.h:56
    template <typename T> T fminT(T a, T b) { return std::fmin(a, b); }
    template <typename T> T fmaxT(T a, T b) { return std::fmax(a, b); }
    template <typename T> T clampT(T f, T lo, T hi) { return fminT(fmaxT(f, lo), hi); }
    template <typename T> T epsT() { return T(std::numeric_limits<float>::epsilon()); } // CR_EPS
    template <typename T> T maxF32T() { return T(3.4028234663852885981170418348452e+38F); }
    template <typename T> T nanT() { return std::numeric_limits<T>::quiet_NaN(); }

    template <typename T>
    V3<T> normalized(V3<T> v) // Vec3::normalize, vec3.h:325-332
    {
        T s = v.sq();
        if (s > 0)
            v = v * rsqrtT(s);
        return v;
    }

    // Quat::rotate / rotateInv (quat.h:117-150)
    template <typename T>
    V3<T> qrot(const T q[4], const V3<T> &v, bool inv)
    {
        const T x = q[0], y = q[1], z = q[2], w = q[3];
        const T vx = T(2) * v.x, vy = T(2) * v.y, vz = T(2) * v.z;
        const T w2 = w * w - T(0.5f);
        const T dot2 = (x * vx + y * vy + z * vz);
        if (!inv)
            return V3<T>((vx * w2 + (y * vz - z * vy) * w + x * dot2), (vy * w2 + (z * vx - x * vz) * w + y * dot2),
                         (vz * w2 + (x * vy - y * vx) * w + z * dot2));
        return V3<T>((vx * w2 - (y * vz - z * vy) * w + x * dot2), (vy * w2 - (z * vx - x * vz) * w + y * dot2),
                     (vz * w2 - (x * vy - y * vx) * w + z * dot2));
    }

    template <typename T> V3<T> ld3(const CrB200Float4 &f) { return V3<T>(T(f.x), T(f.y), T(f.z)); }
    inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

    struct SdfView
    {
        const CrB200Int4 *dim;
        const CrB200Float4 *lbcs;
        const CrB200Float4 *data;
    };

    // Trilinear distance of an SDF grid, with the reference's index pairing (sdf.h:243-276).
    template <typename T>
    T trilinearRef(const SdfView &s, const CrB200Int4 &dim, int offset, int bx, int by, int bz, const V3<T> &frac)
    {
        T vals[8];
        for (int dx = 0; dx <= 1; ++dx)
            for (int dy = 0; dy <= 1; ++dy)
                for (int dz = 0; dz <= 1; ++dz)
                {
                    int idx = (dx << 2) | (dy << 1) | dz;
                    int g = offset + ((bz + dz) * dim.x * dim.y) + ((by + dy) * dim.x) + (bx + dx);
                    vals[idx] = T(s.data[g].w);
                }
        T fx = frac.x, fy = frac.y, fz = frac.z;
        T ox = T(1) - fx, oy = T(1) - fy, oz = T(1) - fz;
        T w[8] = {ox * oy * oz, fx * oy * oz, ox * fy * oz, fx * fy * oz, ox * oy * fz, fx * oy * fz, ox * fy * fz, fx * fy * fz};
        T acc = 0;
        for (int i = 0; i < 8; ++i)
            acc += vals[i] * w[i];
        return acc;
    }

    // getGeometrySdf (sdf.h:67-496).  Returns the spine flag; grad/dist in local units.
    template <typename T>
    bool geometrySdf(const V3<T> &lp, int type, const CrB200Float4 &p0f, const SdfView &s, V3<T> &grad, T &dist,
                     V3<T> *tangent)
    {
        const V3<T> p0(T(p0f.x), T(p0f.y), T(p0f.z));
        bool inSpine = false;
        switch (type)
        {
        case CRB200_GEOM_BOX:
        {
            V3<T> pen = V3<T>(std::fabs(lp.x), std::fabs(lp.y), std::fabs(lp.z)) - p0;
            V3<T> sg(lp.x < 0.0 ? T(-1) : T(1), lp.y < 0.0 ? T(-1) : T(1), lp.z < 0.0 ? T(-1) : T(1));
            T g = fmaxT(pen.x, fmaxT(pen.y, pen.z));
            V3<T> q(fmaxT(pen.x, T(0)), fmaxT(pen.y, T(0)), fmaxT(pen.z, T(0)));
            T l = std::sqrt(q.sq());
            V3<T> dir = (g > 0.0) ? q / l
                                  : ((pen.x > pen.y) ? ((pen.x > pen.z) ? V3<T>(1, 0, 0) : V3<T>(0, 0, 1))
                                                     : ((pen.y > pen.z) ? V3<T>(0, 1, 0) : V3<T>(0, 0, 1)));
            grad = sg.mul(dir);
            dist = l + fminT(g, T(0));
            break;
        }
        case CRB200_GEOM_SPHERE:
        {
            T len = std::sqrt(lp.sq());
            grad = lp / fmaxT(len, epsT<T>());
            dist = len - p0.x;
            break;
        }
        case CRB200_GEOM_PLANE:
            grad = V3<T>(0, 1, 0);
            dist = lp.y;
            break;
        case CRB200_GEOM_CAPSULE:
        {
            const T h2 = p0.y * T(2);
            V3<T> pa = lp;
            pa.y -= p0.y;
            const T h = clampT(-pa.y / h2, T(0.0), T(1.0));
            pa.y += h2 * h;
            const T d = std::sqrt(pa.sq());
            grad = pa / fmaxT(d, epsT<T>());
            dist = d - p0.x;
            break;
        }
        case CRB200_GEOM_ARC:
        {
            T ang = std::atan2(lp.z, lp.x);
            if (ang < p0.x || ang > p0.y)
            {
                grad = V3<T>(0, 1, 0);
                dist = nanT<T>();
                break;
            }
            V3<T> proj(std::cos(ang), 0, std::sin(ang));
            V3<T> ptp = lp - proj;
            T d = std::sqrt(ptp.sq());
            grad = ptp / fmaxT(d, epsT<T>());
            dist = d;
            if (tangent)
                *tangent = V3<T>(-proj.z, 0, proj.x);
            break;
        }
        case CRB200_GEOM_TRIANGLE_MESH:
        {
            const int off = (int)fbits(p0f.x), id = (int)fbits(p0f.y);
            const CrB200Float4 lb = s.lbcs[id];
            const CrB200Int4 dim = s.dim[id];
            V3<T> sp = (lp - ld3<T>(lb)) / T(lb.w);
            int qx = (int)(sp.x + T(0.5f)), qy = (int)(sp.y + T(0.5f)), qz = (int)(sp.z + T(0.5f));
            if (qx < 0 || qx >= dim.x || qy < 0 || qy >= dim.y || qz < 0 || qz >= dim.z)
            {
                grad = V3<T>(0, 1, 0);
                dist = maxF32T<T>();
                break;
            }
            int qi = off + (qz * dim.x * dim.y) + (qy * dim.x) + qx;
            grad = ld3<T>(s.data[qi]);
            int bx = (int)sp.x, by = (int)sp.y, bz = (int)sp.z;
            V3<T> fr(sp.x - T(bx), sp.y - T(by), sp.z - T(bz));
            if (bx < 0 || bx >= dim.x - 1 || by < 0 || by >= dim.y - 1 || bz < 0 || bz >= dim.z - 1)
            {
                dist = T(s.data[qi].w);
                break;
            }
            dist = trilinearRef(s, dim, off, bx, by, bz, fr);
            break;
        }
        case CRB200_GEOM_QUAD_SLICER:
        {
            const T hx = p0.x, hz = p0.y;
            if (lp.x < -hx || lp.x > hx || lp.z < -hz || lp.z > hz)
            {
                grad = V3<T>(0, 0, 0);
                dist = maxF32T<T>();
            }
            else
            {
                grad = V3<T>(0, std::copysign(T(1), lp.y), 0);
                dist = std::fabs(lp.y);
            }
            break;
        }
        case CRB200_GEOM_TRIANGLE_MESH_SLICER:
        {
            grad = V3<T>(0, 1, 0);
            dist = nanT<T>();
            const int off = (int)fbits(p0f.x) + 1, id = (int)fbits(p0f.y);
            const CrB200Float4 lb = s.lbcs[id];
            const CrB200Int4 dim = s.dim[id];
            V3<T> sp = (lp - ld3<T>(lb)) / T(lb.w);
            int qx = (int)(sp.x + T(0.5f)), qy = (int)(sp.y + T(0.5f)), qz = (int)(sp.z + T(0.5f));
            if (qx < 1 || qx >= dim.x - 1 || qy < 1 || qy >= dim.y - 1 || qz < 1 || qz >= dim.z - 1)
                break;
            int qi = off + (qz * dim.x * dim.y) + (qy * dim.x) + qx;
            T qd = T(s.data[qi].w);
            if (std::isnan(qd))
                break;
            grad = ld3<T>(s.data[qi]);
            int bx = (int)sp.x, by = (int)sp.y, bz = (int)sp.z;
            V3<T> fr(sp.x - T(bx), sp.y - T(by), sp.z - T(bz));
            T iv = trilinearRef(s, dim, off, bx, by, bz, fr);
            if (std::isnan(iv))
                break;
            dist = std::fabs(iv);
            if (qd * iv < 0)
                grad = V3<T>(-grad.x, -grad.y, -grad.z);
            const CrB200Float4 spine = s.data[off - 1];
            if (std::isnan(spine.x))
                break;
            V3<T> sn = ld3<T>(spine);
            T len = std::sqrt(sn.sq());
            T side = lp.dot(sn / len) + T(spine.w);
            if (side > 0)
            {
                dist -= len - 1;
                inSpine = true;
            }
            break;
        }
        case CRB200_GEOM_CONNECTED_LINE_SEGMENTS:
        {
            grad = V3<T>(0, 1, 0);
            dist = nanT<T>();
            const int off = (int)fbits(p0f.x), id = (int)fbits(p0f.y), size = (int)fbits(p0f.z);
            V3<T> bmin = ld3<T>(s.lbcs[id]), bmax = ld3<T>(s.data[off]);
            if (lp.x < bmin.x || lp.x > bmax.x || lp.y < bmin.y || lp.y > bmax.y || lp.z < bmin.z || lp.z > bmax.z)
                break;
            int closestIdx = 0;
            V3<T> closest;
            T closestD = maxF32T<T>();
            V3<T> pt0, pt1;
            for (int p = off + 1; p < off + size - 1; ++p)
            {
                pt0 = ld3<T>(s.data[p]);
                pt1 = ld3<T>(s.data[p + 1]);
                V3<T> line = pt1 - pt0;
                V3<T> pv = lp - pt0;
                T t = pv.dot(line) / line.sq();
                t = fmaxT(T(0), fminT(T(1), t));
                V3<T> proj = pt0 + line * t;
                T d = std::sqrt((lp - proj).sq());
                if (d < closestD)
                {
                    closestD = d;
                    closest = proj;
                    closestIdx = p;
                }
            }
            pt0 = ld3<T>(s.data[off + 1]);
            if ((closest - pt0).sq() < epsT<T>() || (closest - pt1).sq() < epsT<T>())
                break;
            grad = normalized(lp - closest);
            if (tangent)
                *tangent = normalized(ld3<T>(s.data[closestIdx]) - ld3<T>(s.data[closestIdx + 1]));
            dist = closestD;
            break;
        }
        default:
            break;
        }
        return inSpine;
    }

    // getGeometryModSdf (sdf.h:504-662): projection flag, signed side distance in dist.
    template <typename T>
    bool geometryModSdf(const V3<T> &lp, int type, const CrB200Float4 &p0f, const SdfView &s, V3<T> &grad, T &dist)
    {
        if (type == CRB200_GEOM_QUAD_SLICER)
        {
            const T hx = T(p0f.x), hz = T(p0f.y);
            if (lp.x < -hx || lp.x > hx || lp.z < -hz || lp.z > hz)
                return false;
            grad = V3<T>(0, std::copysign(T(1), lp.y), 0);
            dist = lp.y;
            return true;
        }
        if (type == CRB200_GEOM_TRIANGLE_MESH_SLICER)
        {
            grad = V3<T>(0, 1, 0);
            dist = nanT<T>();
            int off = (int)fbits(p0f.x);
            const CrB200Float4 spine = s.data[off];
            if (std::isnan(spine.x))
                return false;
            T side = lp.dot(ld3<T>(spine)) + T(spine.w);
            if (side > 0)
                return false;
            off++;
            const int id = (int)fbits(p0f.y);
            const CrB200Float4 lb = s.lbcs[id];
            const CrB200Int4 dim = s.dim[id];
            V3<T> sp = (lp - ld3<T>(lb)) / T(lb.w);
            int qx = (int)(sp.x + T(0.5f)), qy = (int)(sp.y + T(0.5f)), qz = (int)(sp.z + T(0.5f));
            if (qx < 1 || qx >= dim.x - 1 || qy < 1 || qy >= dim.y - 1 || qz < 1 || qz >= dim.z - 1)
                return false;
            int qi = off + (qz * dim.x * dim.y) + (qy * dim.x) + qx;
            T qd = T(s.data[qi].w);
            if (std::isnan(qd))
                return false;
            grad = ld3<T>(s.data[qi]);
            int bx = (int)sp.x, by = (int)sp.y, bz = (int)sp.z;
            V3<T> fr(sp.x - T(bx), sp.y - T(by), sp.z - T(bz));
            T iv = trilinearRef(s, dim, off, bx, by, bz, fr);
            if (std::isnan(iv))
                return false;
            dist = iv;
            if (qd * iv < 0)
                grad = V3<T>(-grad.x, -grad.y, -grad.z);
            return true;
        }
        return false;
    }

    template <typename T>
    struct Solver
    {
        int solverType;
        int nmax;
        V3<T> gmin, gmax;
        T dx, invDx, cellVol;
        int nx, ny, nz, numNodes;
        T dt = T(0.002f);
        V3<T> gravity;
        int iterations = 10;
        int contactModel = 0;

        std::vector<T> x, v, m, F, C, V0, mat;
        std::vector<int> matType;
        std::vector<unsigned char> mask;
        unsigned int numActive = 0;

        std::vector<T> grid;  // 4 per node: momentum/velocity xyz, mass
        std::vector<T> force; // standard MPM node force, 3 per node

        int numShapes = 0;
        std::vector<int> shapeIds;
        CrB200ShapeData sh{};
        CrB200GeometryData ge{};
        SdfView sdf{};
        std::vector<T> coupling; // 6 per shape id: force xyz, torque xyz

        V3<T> X(int p) const { return V3<T>(x[3 * p], x[3 * p + 1], x[3 * p + 2]); }
        V3<T> Vv(int p) const { return V3<T>(v[3 * p], v[3 * p + 1], v[3 * p + 2]); }
        void setX(int p, const V3<T> &a) { x[3 * p] = a.x; x[3 * p + 1] = a.y; x[3 * p + 2] = a.z; }
        void setV(int p, const V3<T> &a) { v[3 * p] = a.x; v[3 * p + 1] = a.y; v[3 * p + 2] = a.z; }
        M3<T> getM(const std::vector<T> &a, int p) const
        {
            M3<T> r;
            r.c0 = V3<T>(a[9 * p + 0], a[9 * p + 1], a[9 * p + 2]);
            r.c1 = V3<T>(a[9 * p + 3], a[9 * p + 4], a[9 * p + 5]);
            r.c2 = V3<T>(a[9 * p + 6], a[9 * p + 7], a[9 * p + 8]);
            return r;
        }
        void setM(std::vector<T> &a, int p, const M3<T> &r)
        {
            for (int c = 0; c < 3; ++c)
                for (int rr = 0; rr < 3; ++rr)
                    a[9 * p + 3 * c + rr] = r(rr, c);
        }
        V3<T> nodeXYZ(int n) const { return V3<T>(grid[4 * n], grid[4 * n + 1], grid[4 * n + 2]); }

        // --------------------------------------------------------------------------------------
        // Weights (shape_functions.h:44-75)
        static void weights(const V3<T> &fx, T w[3][3])
        {
            for (int d = 0; d < 3; ++d)
            {
                w[0][d] = T(0.5f) * std::pow(T(1.5f) - fx[d], T(2));
                w[1][d] = T(0.75f) - std::pow(fx[d] - T(1.0f), T(2));
                w[2][d] = T(0.5f) * std::pow(fx[d] - T(0.5f), T(2));
            }
        }
        static void weightGrads(const V3<T> &fx, T dw[3][3])
        {
            for (int d = 0; d < 3; ++d)
            {
                dw[0][d] = T(fx[d] - 1.5);
                dw[1][d] = T(2.0f) * (T(1.0f) - fx[d]);
                dw[2][d] = fx[d] - T(0.5f);
            }
        }
        // baseCoord and fx (mls_mpm_algorithm.h:170-175)
        void stencil(const V3<T> &pos, int base[3], V3<T> &fx) const
        {
            V3<T> sp = (pos - gmin) * invDx;
            for (int d = 0; d < 3; ++d)
            {
                base[d] = (int)(sp[d] - T(0.5f));
                fx[d] = sp[d] - T(base[d]);
            }
        }
        bool inGrid(int i, int j, int k) const { return i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz; }
        int nodeIndex(int i, int j, int k) const { return i + j * nx + k * nx * ny; }

        // --------------------------------------------------------------------------------------
        // Stress (constitutive_models.h:49-118); returns Kirchhoff stress.
        M3<T> stress(int p, const M3<T> &Fp) const
        {
            const T lambda = mat[4 * p], mu = mat[4 * p + 1];
            const int ty = matType[p];
            M3<T> s;
            if (ty == CRB200_MATERIAL_NEOHOOKEAN)
            {
                T J = Fp.det();
                if (J < 1e-6)
                    J = T(1e-6);
                const M3<T> b = Fp * Fp.T_();
                M3<T> diag;
                T l = lambda * std::log(J);
                diag.c0.x = l; diag.c1.y = l; diag.c2.z = l;
                s = (b - M3<T>::I()) * mu + diag;
            }
            else if (ty == CRB200_MATERIAL_COROTATIONAL || ty == CRB200_MATERIAL_LINEAR_ELASTIC)
            {
                // eCoRotational's own result is discarded by the missing `break` (Q1).
                const M3<T> strain = (Fp.T_() * Fp - M3<T>::I()) * T(0.5f);
                M3<T> diag;
                T tr = strain.trace();
                diag.c0.x = tr * lambda; diag.c1.y = tr * lambda; diag.c2.z = tr * lambda;
                s = diag + strain * (T(2) * mu);
                s = (Fp * s) * Fp.T_();
            }
            return s;
        }

        // --------------------------------------------------------------------------------------
        // Slicer predicate (mpm_rigid_contact.h:401-478).
        bool differentSides(const V3<T> &p1, const V3<T> &p2, V3<T> *normal) const
        {
            for (int si = 0; si < numShapes; ++si)
            {
                const int id = shapeIds[si];
                const int gid = sh.geometryIdx[id];
                const int gt = ge.type[gid];
                if (gt != CRB200_GEOM_QUAD_SLICER && gt != CRB200_GEOM_TRIANGLE_MESH_SLICER)
                    continue;
                const V3<T> pos = ld3<T>(sh.position[id]);
                const T q[4] = {T(sh.rotation[id].x), T(sh.rotation[id].y), T(sh.rotation[id].z), T(sh.rotation[id].w)};
                const V3<T> isc = ld3<T>(sh.invScale[id]);
                V3<T> r1 = qrot(q, p1 - pos, true).mul(isc);
                V3<T> r2 = qrot(q, p2 - pos, true).mul(isc);
                V3<T> g1, g2;
                T d1 = 0, d2 = 0;
                if (!geometryModSdf(r1, gt, ge.params0[gid], sdf, g1, d1))
                    continue;
                bool on2 = geometryModSdf(r2, gt, ge.params0[gid], sdf, g2, d2);
                if (on2 && !(std::signbit(d1) == std::signbit(d2)))
                {
                    if (normal)
                    {
                        V3<T> g = g2.mul(isc);
                        *normal = g * rsqrtT(g.sq());
                    }
                    return true;
                }
            }
            return false;
        }

        // --------------------------------------------------------------------------------------
        // resolveRigidCollision (mpm_rigid_contact.h:101-399).  vel/mass and pos are in-out.
        void rigidCollision(bool isParticle, bool effMass, V3<T> &vel, T mass, V3<T> &pos)
        {
            for (int si = 0; si < numShapes; ++si)
            {
                const int id = shapeIds[si];
                const int stype = sh.type[id];
                const V3<T> isc = ld3<T>(sh.invScale[id]);
                const int gid = sh.geometryIdx[id];
                const int gt = ge.type[gid];
                if (isParticle && (gt == CRB200_GEOM_CONNECTED_LINE_SEGMENTS || gt == CRB200_GEOM_ARC))
                    continue;
                const V3<T> spos = ld3<T>(sh.position[id]);
                const T q[4] = {T(sh.rotation[id].x), T(sh.rotation[id].y), T(sh.rotation[id].z), T(sh.rotation[id].w)};
                V3<T> wrel = pos - spos;
                V3<T> rel = qrot(q, wrel, true);
                V3<T> lp = rel.mul(isc);
                V3<T> grad, tangent;
                T dist = 0;
                bool onSpine = geometrySdf(lp, gt, ge.params0[gid], sdf, grad, dist, &tangent);
                if (std::isnan(dist))
                    continue;
                grad = grad.mul(isc);
                const T is = rsqrtT(grad.sq());
                dist = dist * is;
                grad = grad * is;
                const CrB200Float4 sp0 = sh.params0[id];
                dist -= T(sp0.w);
                T smooth = isParticle ? T(0) : T(sp0.x);
                if (!(dist < smooth))
                    continue;
                V3<T> normal = qrot(q, grad, false);
                V3<T> rigidVel = stype == CRB200_SHAPE_STATIC
                                     ? V3<T>()
                                     : ld3<T>(sh.linearVelocity[id]) + ld3<T>(sh.angularVelocity[id]).cross(wrel);
                V3<T> relVel = vel - rigidVel;
                T vn = relVel.dot(normal);
                V3<T> nComp = normal * vn;
                if (isParticle)
                {
                    T inside = fminT(dist, T(0));
                    V3<T> corr = normal * inside;
                    pos = pos - corr;
                    continue;
                }
                if (vn >= T(0))
                    continue;
                T friction = onSpine ? T(1e2f) : T(sp0.z);
                const T sticky = T(sp0.y);
                V3<T> resp;
                if (effMass && stype == CRB200_SHAPE_DYNAMIC)
                {
                    // mpm_rigid_contact.h:219-301
                    const CrB200Float4 cim = sh.comInvMass[id];
                    const T invMassRigid = T(cim.w);
                    const T rigidMass = invMassRigid > T(0) ? T(1) / invMassRigid : T(0);
                    // A non-positive rigid mass leaves the response at its zero initial value
                    // (Vec3f default constructor), so the node velocity becomes zero (:231, :296).
                    if (!(rigidMass > T(0)))
                    {
                        vel = V3<T>();
                        continue;
                    }
                    const V3<T> r = wrel - qrot(q, ld3<T>(cim), false);
                    V3<T> rxn = r.cross(normal);
                    V3<T> rxnl = qrot(q, rxn, true);
                    const CrB200Float4 i0 = sh.inertiaInv0[id], i1 = sh.inertiaInv1[id];
                    V3<T> wl(T(i0.x) * rxnl.x + T(i1.x) * rxnl.y + T(i1.y) * rxnl.z,
                             T(i1.x) * rxnl.x + T(i0.y) * rxnl.y + T(i1.z) * rxnl.z,
                             T(i1.y) * rxnl.x + T(i1.z) * rxnl.y + T(i0.z) * rxnl.z);
                    V3<T> ww = qrot(q, wl, false);
                    V3<T> tt = ww.cross(r);
                    T invMassRigidN = invMassRigid + normal.dot(tt);
                    T invMassGrid = T(1) / mass;
                    T invMassComb = invMassGrid + invMassRigidN;
                    if (!(invMassComb > T(0)))
                    {
                        vel = V3<T>();
                        continue;
                    }
                    T Jn = T(-1) * vn / invMassComb;
                    V3<T> impN = normal * Jn;
                    V3<T> vt = relVel - (normal * vn);
                    T vtn = std::sqrt(vt.sq());
                    V3<T> impT;
                    if (vtn > epsT<T>())
                    {
                        T stopJt = vtn / invMassComb;
                        T maxJt = friction * Jn;
                        T fJt = fminT(maxJt, stopJt);
                        T left = vtn - (fJt * invMassComb);
                        T fin = left * sticky;
                        T totJt = (vtn - fin) / invMassComb;
                        impT = (vt * T(-1) / vtn) * totJt;
                    }
                    V3<T> tot = impN + impT;
                    resp = vel + (tot * invMassGrid);
                    V3<T> mom = tot * T(-1);
                    addMomentum(id, mom, r);
                }
                else
                {
                    // kinematic view (mpm_rigid_contact.h:304-396; the effective-mass model uses
                    // the same response for non-dynamic shapes, :273-299)
                    V3<T> tang = relVel - nComp;
                    if (gt == CRB200_GEOM_CONNECTED_LINE_SEGMENTS || gt == CRB200_GEOM_ARC)
                    {
                        V3<T> td = normalized(tangent.mul(isc));
                        td = qrot(q, td, false);
                        tang = td * tang.dot(td);
                    }
                    T tn = std::sqrt(tang.sq());
                    T fc = fmaxT(friction * vn / (tn + epsT<T>()), T(-1));
                    resp = tang + tang * fc;
                    resp = resp * sticky;
                    resp = resp + rigidVel;
                    if (!effMass && stype == CRB200_SHAPE_DYNAMIC)
                    {
                        V3<T> mc = vel - resp;
                        mc = mc * mass;
                        addMomentum(id, mc, pos - spos);
                    }
                }
                vel = resp;
            }
        }

        void addMomentum(int id, const V3<T> &mom, const V3<T> &lpos)
        {
            V3<T> tq = lpos.cross(mom);
            T *c = &coupling[6 * id];
            c[0] += mom.x; c[1] += mom.y; c[2] += mom.z;
            c[3] += tq.x; c[4] += tq.y; c[5] += tq.z;
        }

        // --------------------------------------------------------------------------------------
        void resetGrid()
        {
            std::fill(grid.begin(), grid.end(), T(0));
            std::fill(force.begin(), force.end(), T(0));
        }

        // MLS P2G (mls_mpm_algorithm.h:147-241)
        void mlsP2G()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                const V3<T> xp = X(p);
                const T mp = m[p];
                int base[3];
                V3<T> fx;
                stencil(xp, base, fx);
                T w[3][3];
                weights(fx, w);
                V3<T> vp = Vv(p) + gravity * dt;
                setV(p, vp);
                const M3<T> Fp = getM(F, p), Cp = getM(C, p);
                const M3<T> s = stress(p, Fp);
                const T coef = -dt * T(4) * invDx * invDx * V0[p];
                const M3<T> affine = s * coef + Cp * mp;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const V3<T> d = (V3<T>(T(i), T(j), T(k)) - fx) * dx;
                            if (numShapes && differentSides(xp, xp + d, nullptr))
                                continue;
                            const int n = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            const T wt = w[i][0] * w[j][1] * w[k][2];
                            grid[4 * n + 3] += wt * mp;
                            V3<T> c = (vp * mp + affine * d) * wt;
                            grid[4 * n] += c.x; grid[4 * n + 1] += c.y; grid[4 * n + 2] += c.z;
                        }
            }
        }

        // Grid update shared by MLS / PB / standard (mls_mpm_algorithm.h:243-294,
        // pb_mpm_algorithm.h:233-284, standard_mpm_algorithm.h:217-272).
        void updateGrid(T cutoff, bool withForce)
        {
            for (int n = 0; n < numNodes; ++n)
            {
                int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
                T *g = &grid[4 * n];
                if (g[3] < cutoff)
                    continue;
                if (withForce)
                {
                    g[0] += force[3 * n] * dt; g[1] += force[3 * n + 1] * dt; g[2] += force[3 * n + 2] * dt;
                }
                g[0] /= g[3]; g[1] /= g[3]; g[2] /= g[3];
                V3<T> pos = V3<T>(T(i) * dx, T(j) * dx, T(k) * dx) + gmin;
                V3<T> vel(g[0], g[1], g[2]);
                pos = pos + V3<T>(g[0] * dt, g[1] * dt, g[2] * dt);
                rigidCollision(false, contactModel == 1, vel, g[3], pos);
                g[0] = vel.x; g[1] = vel.y; g[2] = vel.z;
                if (i < 2 || i > nx - 3) g[0] = 0;
                if (j < 2 || j > ny - 3) g[1] = 0;
                if (k < 2 || k > nz - 3) g[2] = 0;
            }
        }

        // G2P gather of v and the APIC matrix (mls_mpm_algorithm.h:312-358).
        void gatherVC(int p, const V3<T> &xp, const V3<T> &vkick, V3<T> &vOut, M3<T> &COut)
        {
            int base[3];
            V3<T> fx;
            stencil(xp, base, fx);
            T w[3][3];
            weights(fx, w);
            V3<T> va;
            M3<T> ca;
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    for (int k = 0; k < 3; k++)
                    {
                        if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                            continue;
                        const int n = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                        V3<T> nv = nodeXYZ(n);
                        const V3<T> d = (V3<T>(T(i), T(j), T(k)) - fx) * dx;
                        V3<T> nrm;
                        if (numShapes && differentSides(xp, xp + d, &nrm))
                            nv = vkick - nrm * vkick.dot(nrm) * T(2.0f);
                        const T wt = w[i][0] * w[j][1] * w[k][2];
                        va = va + nv * wt;
                        ca = ca + refOuter(nv * wt, d);
                    }
            vOut = va;
            COut = ca * (T(4) * invDx);
        }

        void clampPos(V3<T> &xp) const
        {
            for (int d = 0; d < 3; ++d)
                xp[d] = fminT(fmaxT(xp[d], gmin[d]), gmax[d]);
        }

        // MLS G2P (mls_mpm_algorithm.h:296-390)
        void mlsG2P()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                V3<T> xp = X(p), vp = Vv(p);
                V3<T> vn;
                M3<T> Cn;
                gatherVC(p, xp, vp, vn, Cn);
                xp = xp + vn * dt;
                clampPos(xp);
                rigidCollision(true, false, vn, m[p], xp);
                M3<T> Fp = getM(F, p);
                Fp.leftMul(M3<T>::I() + Cn * dt);
                setX(p, xp);
                setV(p, vn);
                setM(F, p, Fp);
                setM(C, p, Cn);
            }
        }

        // PB-MPM material constraint (constitutive_models.h:123-156)
        void solveMaterialConstraint(int p, const M3<T> &Fp, M3<T> &Cp) const
        {
            const int ty = matType[p];
            if (ty != CRB200_MATERIAL_NEOHOOKEAN && ty != CRB200_MATERIAL_COROTATIONAL)
                return;
            M3<T> tF = (M3<T>::I() + Cp * dt) * Fp;
            T A[9];
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                    A[c * 3 + r] = tF(r, c);
            Svd3<T> sv;
            svd3(A, sv);
            M3<T> U, Vm;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                {
                    U.at(r, c) = sv.U[c * 3 + r];
                    Vm.at(r, c) = sv.V[c * 3 + r];
                }
            const T detF = tF.det();
            const T cd = clampT(T(std::fabs(detF)), T(0.1f), T(1000.0f));
            const M3<T> Q = tF * (T(1.0f) / (std::copysign(T(1.0f), detF) * std::sqrt(cd)));
            const T ratio = mat[4 * p + 1];
            // svd3 hands the column-major matrix to a row-major SVD (svd3.h:1271-1274), so the
            // reference's `u * vt` is the polar rotation of targetF^T, i.e. R^T = V U^T.
            tF = (Vm * U.T_()) * ratio + Q * (T(1.0f) - ratio);
            const T relax = mat[4 * p];
            Cp = Cp + ((tF * Fp.inverse() - M3<T>::I()) - Cp * dt) * relax;
        }

        // PB P2G (pb_mpm_algorithm.h:150-231)
        void pbP2G()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                const V3<T> xp = X(p), vp = Vv(p);
                const T mp = m[p];
                M3<T> Cp = getM(C, p);
                solveMaterialConstraint(p, getM(F, p), Cp);
                setM(C, p, Cp);
                int base[3];
                V3<T> fx;
                stencil(xp, base, fx);
                T w[3][3];
                weights(fx, w);
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const V3<T> d = (V3<T>(T(i), T(j), T(k)) - fx) * dx;
                            if (numShapes && differentSides(xp, xp + d, nullptr))
                                continue;
                            const int n = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            const T wt = w[i][0] * w[j][1] * w[k][2];
                            const T wm = wt * mp;
                            grid[4 * n + 3] += wm;
                            V3<T> c = (vp + Cp * d) * wm;
                            grid[4 * n] += c.x; grid[4 * n + 1] += c.y; grid[4 * n + 2] += c.z;
                        }
            }
        }

        // PB G2P (pb_mpm_algorithm.h:286-361): v and C only
        void pbG2P()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                V3<T> vn;
                M3<T> Cn;
                gatherVC(p, X(p), Vv(p), vn, Cn);
                setV(p, vn);
                setM(C, p, Cn);
            }
        }

        // PB integrate (pb_mpm_algorithm.h:363-408)
        void pbIntegrate()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                V3<T> xp = X(p), vp = Vv(p);
                xp = xp + vp * dt;
                clampPos(xp);
                vp = vp + gravity * dt;
                rigidCollision(true, false, vp, m[p], xp);
                M3<T> Fp = getM(F, p);
                Fp.leftMul(M3<T>::I() + getM(C, p) * dt);
                setX(p, xp);
                setV(p, vp);
                setM(F, p, Fp);
            }
        }

        // Standard P2G (standard_mpm_algorithm.h:146-215): every index below numActive.
        void stdP2G()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                const V3<T> xp = X(p), vp = Vv(p);
                const T mp = m[p];
                int base[3];
                V3<T> fx;
                stencil(xp, base, fx);
                T w[3][3], dw[3][3];
                weights(fx, w);
                weightGrads(fx, dw);
                const M3<T> s = stress(p, getM(F, p));
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const int n = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            const T wt = w[i][0] * w[j][1] * w[k][2];
                            const V3<T> gw(dw[i][0] * w[j][1] * w[k][2], w[i][0] * dw[j][1] * w[k][2],
                                           w[i][0] * w[j][1] * dw[k][2]);
                            const V3<T> ext = gravity * (wt * mp);
                            const V3<T> in = (s * gw) * (-V0[p]);
                            grid[4 * n + 3] += wt * mp;
                            V3<T> mv = vp * (wt * mp);
                            grid[4 * n] += mv.x; grid[4 * n + 1] += mv.y; grid[4 * n + 2] += mv.z;
                            V3<T> f = ext + in;
                            force[3 * n] += f.x; force[3 * n + 1] += f.y; force[3 * n + 2] += f.z;
                        }
            }
        }

        // Standard G2P (standard_mpm_algorithm.h:274-352)
        void stdG2P()
        {
            for (int p = 0; p < (int)numActive; ++p)
            {
                if (!mask[p])
                    continue;
                V3<T> xp = X(p);
                int base[3];
                V3<T> fx;
                stencil(xp, base, fx);
                T w[3][3], dw[3][3];
                weights(fx, w);
                weightGrads(fx, dw);
                V3<T> va;
                M3<T> gv;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const int n = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            const T wt = w[i][0] * w[j][1] * w[k][2];
                            const V3<T> nv = nodeXYZ(n);
                            va = va + nv * wt;
                            const V3<T> gw(dw[i][0] * w[j][1] * w[k][2], w[i][0] * dw[j][1] * w[k][2],
                                           w[i][0] * w[j][1] * dw[k][2]);
                            gv = gv + refOuter(gw, nv);
                        }
                V3<T> vn = va;
                xp = xp + va * dt;
                clampPos(xp);
                rigidCollision(true, false, vn, m[p], xp);
                M3<T> Fp = getM(F, p);
                Fp.leftMul(M3<T>::I() + gv * dt);
                setX(p, xp);
                setV(p, vn);
                setM(F, p, Fp);
            }
        }

        // computeInitialData (mls_mpm_algorithm.h:46-145, cpu_mls_mpm_solver.cpp:63-96):
        // scatters into the live grid like the reference.
        void initialData(unsigned n, const unsigned *idx)
        {
            for (unsigned ii = 0; ii < n; ++ii)
            {
                int p = (int)idx[ii];
                setM(F, p, M3<T>::I());
                int base[3];
                V3<T> fx;
                stencil(X(p), base, fx);
                T w[3][3];
                weights(fx, w);
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const int nn = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            grid[4 * nn + 3] += (w[i][0] * w[j][1] * w[k][2]) * m[p];
                        }
            }
            for (unsigned ii = 0; ii < n; ++ii)
            {
                int p = (int)idx[ii];
                int base[3];
                V3<T> fx;
                stencil(X(p), base, fx);
                T w[3][3];
                weights(fx, w);
                T dens = 0;
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const int nn = nodeIndex(base[0] + i, base[1] + j, base[2] + k);
                            const T wt = w[i][0] * w[j][1] * w[k][2];
                            dens += (grid[4 * nn + 3] / cellVol) * wt;
                        }
                V0[p] = dens > T(1e-8f) ? m[p] / dens : T(1e-8f);
            }
        }

        void step()
        {
            if (solverType == CRB200_SOLVER_GPU_MLS)
            {
                resetGrid(); mlsP2G(); updateGrid(T(1e-4f), false); mlsG2P();
            }
            else if (solverType == CRB200_SOLVER_GPU_PB)
            {
                for (int it = 0; it < iterations; ++it)
                {
                    resetGrid(); pbP2G(); updateGrid(T(1e-8f), false); pbG2P();
                }
                pbIntegrate();
            }
            else
            {
                resetGrid(); stdP2G(); updateGrid(T(1e-4f), true); stdG2P();
            }
        }

        void phase(int ph)
        {
            const bool mls = solverType == CRB200_SOLVER_GPU_MLS, pb = solverType == CRB200_SOLVER_GPU_PB;
            switch (ph)
            {
            case 0: resetGrid(); break;
            case 1: mls ? mlsP2G() : pb ? pbP2G() : stdP2G(); break;
            case 2: updateGrid(pb ? T(1e-8f) : T(1e-4f), !mls && !pb); break;
            case 3: mls ? mlsG2P() : pb ? pbG2P() : stdG2P(); break;
            case 4: if (pb) pbIntegrate(); break;
            }
        }
    };

    struct Handle
    {
        int prec;
        void *s;
    };

    template <typename T>
    Solver<T> *create(int solverType, int nmax, float cellSize, const float *mn, const float *mx)
    {
        auto *s = new Solver<T>();
        s->solverType = solverType;
        s->nmax = nmax;
        // Node counts in float exactly like the reference constructor (gpu_mls_mpm_solver.cu:48-49).
        float sz[3], dims[3];
        for (int d = 0; d < 3; ++d)
        {
            sz[d] = mx[d] - mn[d];
            dims[d] = sz[d] / cellSize + 1.0f;
        }
        s->nx = (int)dims[0];
        s->ny = (int)dims[1];
        s->nz = (int)dims[2];
        s->numNodes = s->nx * s->ny * s->nz;
        s->gmin = V3<T>(T(mn[0]), T(mn[1]), T(mn[2]));
        s->gmax = V3<T>(T(mx[0]), T(mx[1]), T(mx[2]));
        s->dx = T(cellSize);
        s->invDx = sizeof(T) == 4 ? T(1 / cellSize) : T(1) / T(cellSize);
        s->cellVol = sizeof(T) == 4 ? T(cellSize * cellSize * cellSize) : T(cellSize) * T(cellSize) * T(cellSize);
        s->x.assign(3 * nmax, 0); s->v.assign(3 * nmax, 0); s->m.assign(nmax, 0);
        s->F.assign(9 * nmax, 0); s->C.assign(9 * nmax, 0); s->V0.assign(nmax, 0);
        s->mat.assign(4 * nmax, 0); s->matType.assign(nmax, 0); s->mask.assign(nmax, 0);
        s->grid.assign(4 * s->numNodes, 0);
        s->force.assign(3 * s->numNodes, 0);
        return s;
    }
} // namespace orc

using namespace orc;

#define DISPATCH(h, ...)                                                                  \
    do                                                                                    \
    {                                                                                     \
        Handle *hh = static_cast<Handle *>(h);                                            \
        if (hh->prec == 64) { auto *s = static_cast<Solver<double> *>(hh->s); __VA_ARGS__; } \
        else { auto *s = static_cast<Solver<float> *>(hh->s); __VA_ARGS__; }              \
    } while (0)

extern "C"
{
    // prec: 32 (reference order, single precision) or 64 (FP64 oracle).
    void *orc_create(int prec, int solverType, int nmax, float cellSize, const float *mn, const float *mx)
    {
        Handle *h = new Handle();
        h->prec = prec;
        if (prec == 64)
            h->s = create<double>(solverType, nmax, cellSize, mn, mx);
        else
            h->s = create<float>(solverType, nmax, cellSize, mn, mx);
        return h;
    }

    void orc_destroy(void *h)
    {
        DISPATCH(h, delete s);
        delete static_cast<Handle *>(h);
    }

    void orc_grid_dims(void *h, int *out) { DISPATCH(h, { out[0] = s->nx; out[1] = s->ny; out[2] = s->nz; }); }

    void orc_set_params(void *h, float dt, const float *g, int iterations, int contactModel)
    {
        DISPATCH(h, {
            using T = std::remove_reference_t<decltype(s->dt)>;
            s->dt = T(dt);
            s->gravity = V3<T>(T(g[0]), T(g[1]), T(g[2]));
            s->iterations = iterations;
            s->contactModel = contactModel;
        });
    }

    // Any pointer may be NULL (keep current).  posMass4: x, y, z, m per particle; vel4: x, y, z, _;
    // F9/C9 column-major; matParams4; matType; mask.
    void orc_set_state(void *h, unsigned n, const double *posMass4, const double *vel4, const double *F9,
                       const double *C9, const double *V0, const double *matParams4, const int *matType,
                       const unsigned char *mask, unsigned numActive)
    {
        DISPATCH(h, {
            using T = std::remove_reference_t<decltype(s->dt)>;
            for (unsigned p = 0; p < n; ++p)
            {
                if (posMass4)
                {
                    for (int d = 0; d < 3; ++d) s->x[3 * p + d] = T(posMass4[4 * p + d]);
                    s->m[p] = T(posMass4[4 * p + 3]);
                }
                if (vel4) for (int d = 0; d < 3; ++d) s->v[3 * p + d] = T(vel4[4 * p + d]);
                if (F9) for (int d = 0; d < 9; ++d) s->F[9 * p + d] = T(F9[9 * p + d]);
                if (C9) for (int d = 0; d < 9; ++d) s->C[9 * p + d] = T(C9[9 * p + d]);
                if (V0) s->V0[p] = T(V0[p]);
                if (matParams4) for (int d = 0; d < 4; ++d) s->mat[4 * p + d] = T(matParams4[4 * p + d]);
                if (matType) s->matType[p] = matType[p];
                if (mask) s->mask[p] = mask[p];
            }
            s->numActive = numActive;
        });
    }

    void orc_get_state(void *h, unsigned n, double *posMass4, double *vel4, double *F9, double *C9, double *V0)
    {
        DISPATCH(h, {
            for (unsigned p = 0; p < n; ++p)
            {
                if (posMass4)
                {
                    for (int d = 0; d < 3; ++d) posMass4[4 * p + d] = double(s->x[3 * p + d]);
                    posMass4[4 * p + 3] = double(s->m[p]);
                }
                if (vel4)
                {
                    for (int d = 0; d < 3; ++d) vel4[4 * p + d] = double(s->v[3 * p + d]);
                    vel4[4 * p + 3] = 0;
                }
                if (F9) for (int d = 0; d < 9; ++d) F9[9 * p + d] = double(s->F[9 * p + d]);
                if (C9) for (int d = 0; d < 9; ++d) C9[9 * p + d] = double(s->C[9 * p + d]);
                if (V0) V0[p] = double(s->V0[p]);
            }
        });
    }

    // Host pointers; shape force/torque outputs are accumulated internally (orc_get_coupling).
    void orc_bind_shapes(void *h, int numShapes, const int *shapeIds, const CrB200ShapeData *shapes,
                         const CrB200GeometryData *geoms, const CrB200GeometrySdfData *sdf)
    {
        DISPATCH(h, {
            s->numShapes = numShapes;
            s->shapeIds.assign(shapeIds, shapeIds + numShapes);
            s->sh = *shapes;
            s->ge = *geoms;
            s->sdf = SdfView{sdf->dimension, sdf->lowerBoundCellSize, sdf->gradientSignedDistance};
            s->coupling.assign(6 * (shapes->size > 0 ? shapes->size : 1), 0);
        });
    }

    void orc_get_coupling(void *h, int shapeId, double *out6)
    {
        DISPATCH(h, { for (int d = 0; d < 6; ++d) out6[d] = double(s->coupling[6 * shapeId + d]); });
    }

    void orc_reset_coupling(void *h) { DISPATCH(h, std::fill(s->coupling.begin(), s->coupling.end(), 0)); }

    void orc_compute_initial_data(void *h, unsigned n, const unsigned *idx) { DISPATCH(h, s->initialData(n, idx)); }
    void orc_step(void *h) { DISPATCH(h, s->step()); }
    void orc_phase(void *h, int phase) { DISPATCH(h, s->phase(phase)); }

    void orc_get_grid(void *h, double *out4, double *force3)
    {
        DISPATCH(h, {
            for (int i = 0; i < 4 * s->numNodes; ++i) out4[i] = double(s->grid[i]);
            if (force3) for (int i = 0; i < 3 * s->numNodes; ++i) force3[i] = double(s->force[i]);
        });
    }

    void orc_set_grid(void *h, const double *in4)
    {
        DISPATCH(h, {
            using T = std::remove_reference_t<decltype(s->dt)>;
            for (int i = 0; i < 4 * s->numNodes; ++i) s->grid[i] = T(in4[i]);
        });
    }

    // Cut masks exactly as P2G evaluates them (bit i*9 + j*3 + k).
    void orc_cut_masks(void *h, unsigned *out)
    {
        DISPATCH(h, {
            using T = std::remove_reference_t<decltype(s->dt)>;
            for (int p = 0; p < (int)s->numActive; ++p)
            {
                unsigned msk = 0;
                const V3<T> xp = s->X(p);
                int base[3];
                V3<T> fx;
                s->stencil(xp, base, fx);
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++)
                        for (int k = 0; k < 3; k++)
                        {
                            if (!s->inGrid(base[0] + i, base[1] + j, base[2] + k))
                                continue;
                            const V3<T> d = (V3<T>(T(i), T(j), T(k)) - fx) * s->dx;
                            if (s->differentSides(xp, xp + d, nullptr))
                                msk |= 1u << (i * 9 + j * 3 + k);
                        }
                out[p] = msk;
            }
        });
    }

    void orc_sdf_query(int prec, int geomType, const float *params0, const CrB200GeometrySdfData *sdfData, int n,
                       const double *localPts4, double *out4, double *tangent4, int *spine)
    {
        SdfView sv{sdfData->dimension, sdfData->lowerBoundCellSize, sdfData->gradientSignedDistance};
        CrB200Float4 p0{params0[0], params0[1], params0[2], params0[3]};
        for (int i = 0; i < n; ++i)
        {
            if (prec == 64)
            {
                V3<double> lp(localPts4[4 * i], localPts4[4 * i + 1], localPts4[4 * i + 2]), g, t;
                double d = 0;
                spine[i] = geometrySdf(lp, geomType, p0, sv, g, d, &t);
                out4[4 * i] = g.x; out4[4 * i + 1] = g.y; out4[4 * i + 2] = g.z; out4[4 * i + 3] = d;
                tangent4[4 * i] = t.x; tangent4[4 * i + 1] = t.y; tangent4[4 * i + 2] = t.z; tangent4[4 * i + 3] = 0;
            }
            else
            {
                V3<float> lp(float(localPts4[4 * i]), float(localPts4[4 * i + 1]), float(localPts4[4 * i + 2])), g, t;
                float d = 0;
                spine[i] = geometrySdf(lp, geomType, p0, sv, g, d, &t);
                out4[4 * i] = g.x; out4[4 * i + 1] = g.y; out4[4 * i + 2] = g.z; out4[4 * i + 3] = d;
                tangent4[4 * i] = t.x; tangent4[4 * i + 1] = t.y; tangent4[4 * i + 2] = t.z; tangent4[4 * i + 3] = 0;
            }
        }
    }

    void orc_svd3(int prec, int n, const double *A9, double *U9, double *V9, double *S3)
    {
        for (int p = 0; p < n; ++p)
        {
            if (prec == 64)
            {
                Svd3<double> o;
                svd3(A9 + 9 * p, o);
                for (int i = 0; i < 9; ++i) { U9[9 * p + i] = o.U[i]; V9[9 * p + i] = o.V[i]; }
                for (int i = 0; i < 3; ++i) S3[3 * p + i] = o.s[i];
            }
            else
            {
                float A[9];
                for (int i = 0; i < 9; ++i) A[i] = float(A9[9 * p + i]);
                Svd3<float> o;
                svd3(A, o);
                for (int i = 0; i < 9; ++i) { U9[9 * p + i] = o.U[i]; V9[9 * p + i] = o.V[i]; }
                for (int i = 0; i < 3; ++i) S3[3 * p + i] = o.s[i];
            }
        }
    }
}
