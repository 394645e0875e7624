/*
 * aslb_asl.hpp -- ASL's C++ API for the lattice-Boltzmann path, over the C ABI
 * of libaslb.so (aslb.h). Header-only.
 *
 * A program written against the Advanced Simulation Library (ASL) for its
 * LBGK path includes ASL's headers by their ASL names (<num/aslLBGK.h>,
 * <num/aslLBGKBC.h>, <aslDataInc.h>, <aslGeomInc.h>, <math/aslTemplates.h>,
 * <acl/aclGenerators.h>, <writers/aslVTKFormatWriters.h>,
 * <utilities/aslTimer.h>, <utilities/aslParametersManager.h>, ...); with
 * -I <repo>/include/asl -I <repo>/include those resolve to thin headers that
 * include this file, and the program links against libaslb.so. The classes
 * and functions keep ASL's names, signatures and ownership (everything is a
 * std::shared_ptr); citations give the reference declaration each follows
 * (paths inside AvtechScientific/ASL).
 *
 * What differs from ASL, by design:
 *  - Data containers (DataWithGhostNodesACLData) hold their values on the
 *    host; the LBGK's density and velocity are views that read the device
 *    fields back (synchronising) whenever their values are asked for, which
 *    is ASL's blocking map-on-read behaviour (src/acl/DataTypes/
 *    aclMemBlock.cxx:111-136). Maps and initial fields are handed to the
 *    library as host arrays when a condition is initialised.
 *  - acl::VectorOfElements is a constant (with the type that selects FP32 or
 *    FP64 storage, src/num/aslLBGK.cxx:125) or a reference to a data
 *    container; there is no expression engine.
 *  - Boundary conditions build their link lists in init() (initAll), from
 *    the map as it stands then.
 *  - Errors throw std::logic_error("ASL ERROR: ...") like ASL's errorMessage
 *    (src/aslUtilities.cxx:68-95), carrying the library's message.
 * Extensions (no ASL counterpart) are marked as such.
 */
#ifndef ASLB_ASL_HPP
#define ASLB_ASL_HPP

#include <aslb.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace asl {

// ---- errors ---------------------------------------------------------------

[[noreturn]] inline void errorMessage(const std::string& msg) { throw std::logic_error("ASL ERROR: " + msg); }

namespace aslb_detail {
inline void check(int rc, const std::string& what) {
  if (rc != ASLB_OK) errorMessage(what + ": " + aslb_last_error());
}
}  // namespace aslb_detail

// ---- AVec (src/math/aslVectorsDynamicLength.h:39-63) ------------------------

template <typename T = double>
class AVec {
  std::vector<T> x_;
  unsigned int n_ = 0;

 public:
  AVec() {}
  explicit AVec(unsigned int s) : x_(s, T(0)), n_(s) {}
  AVec(unsigned int s, T a) : x_(s, a), n_(s) {}
  template <typename Tv>
  explicit AVec(const AVec<Tv>& a) : x_(a.getSize()), n_(a.getSize()) {
    for (unsigned int i = 0; i < n_; ++i) x_[i] = T(a[i]);
  }
  AVec(const AVec&) = default;
  AVec& operator=(const AVec&) = default;
  template <typename Tv>
  const AVec<T>& operator=(const AVec<Tv>& a) {
    resize(a.getSize());
    for (unsigned int i = 0; i < n_; ++i) x_[i] = T(a[i]);
    return *this;
  }
  template <typename Tv>
  const AVec<T>& operator=(const std::vector<Tv>& a) {
    resize((unsigned int)a.size());
    for (unsigned int i = 0; i < n_; ++i) x_[i] = T(a[i]);
    return *this;
  }
  T& operator[](unsigned int i) { return x_[i]; }
  const T& operator[](unsigned int i) const { return x_[i]; }
  const unsigned int& getSize() const { return n_; }
  void resize(unsigned int s) {
    x_.resize(s);
    n_ = s;
  }
};

template <typename T> inline AVec<T> makeAVec(T a1) { return AVec<T>(1, a1); }
template <typename T> inline AVec<T> makeAVec(T a1, T a2) {
  AVec<T> v(2);
  v[0] = a1;
  v[1] = a2;
  return v;
}
template <typename T> inline AVec<T> makeAVec(T a1, T a2, T a3) {
  AVec<T> v(3);
  v[0] = a1;
  v[1] = a2;
  v[2] = a3;
  return v;
}
template <typename T> inline AVec<T> makeAVec(T a1, T a2, T a3, T a4) {
  AVec<T> v(4);
  v[0] = a1;
  v[1] = a2;
  v[2] = a3;
  v[3] = a4;
  return v;
}
template <typename T> inline const unsigned int nD(const AVec<T>& a) { return a.getSize(); }

// Operations of src/math/aslVectorsDynamicLengthOperations.h:43-136: a * b of
// two vectors is the scalar product.
template <typename T> inline const AVec<T> operator+(const AVec<T>& a, const AVec<T>& b) {
  AVec<T> r(a);
  for (unsigned int i = 0; i < a.getSize(); ++i) r[i] += b[i];
  return r;
}
template <typename T> inline const AVec<T> operator-(const AVec<T>& a, const AVec<T>& b) {
  AVec<T> r(a);
  for (unsigned int i = 0; i < a.getSize(); ++i) r[i] -= b[i];
  return r;
}
template <typename T> inline const AVec<T> operator-(const AVec<T>& a) {
  AVec<T> r(a);
  for (unsigned int i = 0; i < a.getSize(); ++i) r[i] = -r[i];
  return r;
}
template <typename T> inline const T operator*(const AVec<T>& a, const AVec<T>& b) {
  T s = T(0);
  for (unsigned int i = 0; i < a.getSize(); ++i) s += a[i] * b[i];
  return s;
}
template <typename T> inline const AVec<T> operator*(const AVec<T>& a, const T& b) {
  AVec<T> r(a);
  for (unsigned int i = 0; i < a.getSize(); ++i) r[i] *= b;
  return r;
}
template <typename T> inline const AVec<T> operator*(const T& a, const AVec<T>& b) { return b * a; }
template <typename T> inline const AVec<T> operator/(const AVec<T>& a, const T& b) {
  AVec<T> r(a);
  for (unsigned int i = 0; i < a.getSize(); ++i) r[i] /= b;
  return r;
}
template <typename T> inline const AVec<T>& operator+=(AVec<T>& a, const AVec<T>& b) { return a = a + b; }
template <typename T> inline const AVec<T>& operator-=(AVec<T>& a, const AVec<T>& b) { return a = a - b; }
template <typename T> inline const AVec<T>& operator*=(AVec<T>& a, const T& b) { return a = a * b; }
template <typename T> inline const bool operator==(const AVec<T>& a, const AVec<T>& b) {
  if (a.getSize() != b.getSize()) return false;
  for (unsigned int i = 0; i < a.getSize(); ++i)
    if (a[i] != b[i]) return false;
  return true;
}
template <typename T> inline const bool operator!=(const AVec<T>& a, const AVec<T>& b) { return !(a == b); }
template <typename T> inline const T l2(const AVec<T>& a) { return a * a; }
template <typename T> inline const AVec<> normalize(const AVec<T>& a) {
  return AVec<>(a) / std::sqrt(double(l2(a)));
}
template <typename T> inline const AVec<T> crossProduct(const AVec<T>& a, const AVec<T>& b) {
  return makeAVec(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
template <typename T> inline const T minComponent(const AVec<T>& a) {
  T m = a[0];
  for (unsigned int i = 1; i < a.getSize(); ++i) m = std::min(m, a[i]);
  return m;
}
template <typename T> inline const T maxComponent(const AVec<T>& a) {
  T m = a[0];
  for (unsigned int i = 1; i < a.getSize(); ++i) m = std::max(m, a[i]);
  return m;
}
template <typename T> inline T sumOfElements(const AVec<T>& a) {
  T s = T(0);
  for (unsigned int i = 0; i < a.getSize(); ++i) s += a[i];
  return s;
}
template <typename T> inline T productOfElements(const AVec<T>& a) {
  T s = T(1);
  for (unsigned int i = 0; i < a.getSize(); ++i) s *= a[i];
  return s;
}
template <typename T> inline std::ostream& operator<<(std::ostream& o, const AVec<T>& a) {
  for (unsigned int i = 0; i < a.getSize(); ++i) o << a[i] << (i + 1 < a.getSize() ? " " : "");
  return o;
}

// ---- Block (src/data/aslBlocks.h:52-130) ------------------------------------

inline AVec<int> castTransformVector(const AVec<int>& s) {
  const unsigned int n = s.getSize();
  AVec<int> r(n, 1);
  int a = 1;
  for (unsigned int i = 0; i + 1 < n; ++i) {
    a *= s[n - 1 - i];
    r[n - 2 - i] = a;
  }
  return r;
}

class Block {
 public:
  typedef AVec<int> DV;
  typedef AVec<> V;

 private:
  DV size;

 public:
  V position;
  double dx;
  DV c2iTransformVector;
  Block() : size(3, 1), position(3, 0.), dx(1.), c2iTransformVector(castTransformVector(size)) {}
  explicit Block(unsigned int nd) : size(nd, 1), position(nd, 0.), dx(1.), c2iTransformVector(castTransformVector(size)) {}
  Block(const DV& s, double dx_, const V& p) : size(s), position(p), dx(dx_), c2iTransformVector(castTransformVector(s)) {}
  explicit Block(const DV& s, double dx_ = 1)
      : size(s), position(s.getSize(), 0.), dx(dx_), c2iTransformVector(castTransformVector(s)) {}
  int c2i(const DV& c) const { return c * c2iTransformVector; }
  void setSize(const DV& s) {
    size = s;
    c2iTransformVector = castTransformVector(s);
  }
  const DV& getSize() const { return size; }
  // position of the corner diagonal to cell (0, 0, 0)
  const V getBPosition() const { return position + V(size - DV(size.getSize(), 1)) * dx; }
};

inline const unsigned int nD(const Block& b) { return b.getSize().getSize(); }

// The block grown (a > 0) or shrunk (a < 0) by a cells on every side
// (src/data/aslBlocks.cxx:30-40).
inline const Block offset(const Block& bl, int a = 1) {
  if (minComponent(bl.getSize()) < -a * 2) errorMessage("The inset is larger than the block size");
  Block b(nD(bl));
  b.position = bl.position - Block::V(nD(bl), a * bl.dx);
  b.setSize(bl.getSize() + Block::DV(nD(bl), a * 2));
  b.dx = bl.dx;
  return b;
}

// ---- velocity sets (src/math/aslTemplates.h, aslTemplates.cxx:146-200) -------

class VectorTemplate {
 public:
  std::vector<AVec<int>> vectors;
  std::vector<double> quasiparticlesCoefs;  // weights
  std::vector<unsigned int> invertVectors;  // opposite directions
  unsigned int dimNumber = 3;
  int q = 0;
  explicit VectorTemplate(int q_) : q(q_) {
    std::vector<int> c(3 * q);
    std::vector<double> w(q);
    std::vector<int> inv(q);
    aslb_detail::check(aslb_lattice(q, c.data(), w.data(), inv.data()), "VectorTemplate");
    for (int i = 0; i < q; ++i) {
      vectors.push_back(makeAVec(c[3 * i], c[3 * i + 1], c[3 * i + 2]));
      quasiparticlesCoefs.push_back(w[i]);
      invertVectors.push_back((unsigned int)inv[i]);
    }
  }
};

inline const VectorTemplate& d3q15() {
  static const VectorTemplate t(15);
  return t;
}
inline const VectorTemplate& d3q19() {
  static const VectorTemplate t(19);
  return t;
}
// With the standard D3Q27 weights: the reference's d3q27() has none
// (src/math/aslTemplates.cxx:187-200).
inline const VectorTemplate& d3q27() {
  static const VectorTemplate t(27);
  return t;
}

}  // namespace asl

// ---- acl: element types and constants (src/acl/aclTypes.h, aclGenerators.h) --

namespace asl {
class AbstractData;
}

namespace acl {

enum TypeID { TYPE_INT, TYPE_UINT, TYPE_FLOAT, TYPE_DOUBLE, TYPE_LONG };
template <typename T> inline TypeID typeToTypeID();
template <> inline TypeID typeToTypeID<int>() { return TYPE_INT; }
template <> inline TypeID typeToTypeID<unsigned int>() { return TYPE_UINT; }
template <> inline TypeID typeToTypeID<float>() { return TYPE_FLOAT; }
template <> inline TypeID typeToTypeID<double>() { return TYPE_DOUBLE; }
template <> inline TypeID typeToTypeID<long>() { return TYPE_LONG; }

// A parameter of the numerics: constants with their element type, or the
// values of a data container.
class VectorOfElements {
 public:
  std::vector<double> constants;
  TypeID type = TYPE_DOUBLE;
  std::shared_ptr<asl::AbstractData> data;
  VectorOfElements() {}
  template <class D, class = decltype(std::declval<D&>().getEContainerSize())>
  VectorOfElements(std::shared_ptr<D> d) : data(std::static_pointer_cast<asl::AbstractData>(d)) {}
  unsigned int size() const;
  bool isConstant() const { return !data; }
  double value(unsigned int i = 0) const {
    if (data) asl::errorMessage("VectorOfElements: a data container is not a constant");
    if (i >= constants.size()) asl::errorMessage("VectorOfElements: component out of range");
    return constants[i];
  }
};

template <typename T> inline VectorOfElements generateVEConstant(T a) {
  VectorOfElements v;
  v.constants = {double(a)};
  v.type = typeToTypeID<T>();
  return v;
}
template <typename T> inline VectorOfElements generateVEConstant(T a, T b) {
  VectorOfElements v;
  v.constants = {double(a), double(b)};
  v.type = typeToTypeID<T>();
  return v;
}
template <typename T> inline VectorOfElements generateVEConstant(T a, T b, T c) {
  VectorOfElements v;
  v.constants = {double(a), double(b), double(c)};
  v.type = typeToTypeID<T>();
  return v;
}
template <typename T> inline VectorOfElements generateVEConstant(const asl::AVec<T>& a) {
  VectorOfElements v;
  for (unsigned int i = 0; i < a.getSize(); ++i) v.constants.push_back(double(a[i]));
  v.type = typeToTypeID<T>();
  return v;
}

}  // namespace acl

namespace asl {

// ---- data containers (src/data/aslDataWithGhostNodes.h:97-145,
//      src/aslGenerators.h) -----------------------------------------------------

// Values of a block with a ghost layer, nComponents arrays of the ghosted
// block, z fastest (ASL's layout). Held on the host; a container bound to a
// device field (the LBGK's density and velocity) reads it back when its
// values are asked for.
class AbstractData {
 protected:
  Block internal_;
  unsigned int ncomp_;
  unsigned int ghost_;
  acl::TypeID type_;
  mutable std::vector<double> values_;
  std::function<void(std::vector<double>&)> pull_;

 public:
  AbstractData(const Block& b, unsigned int ncomp, unsigned int ghost, acl::TypeID type)
      : internal_(b), ncomp_(ncomp), ghost_(ghost), type_(type) {
    values_.assign((size_t)ncomp * cells(), 0.0);
  }
  virtual ~AbstractData() {}
  const Block getBlock() const { return offset(internal_, (int)ghost_); }
  const Block& getInternalBlock() const { return internal_; }
  unsigned int getEContainerSize() const { return ncomp_; }
  unsigned int getGhostLayer() const { return ghost_; }
  acl::TypeID getTypeID() const { return type_; }
  size_t cells() const {
    size_t n = 1;
    for (unsigned int a = 0; a < nD(internal_); ++a) n *= (size_t)(internal_.getSize()[a] + 2 * (int)ghost_);
    return n;
  }
  // host values, component-major; refreshed from the device for bound fields
  std::vector<double>& values() const {
    if (pull_) pull_(values_);
    return values_;
  }
  void bind(std::function<void(std::vector<double>&)> pull) { pull_ = std::move(pull); }
  bool bound() const { return bool(pull_); }
  // FP32 copy of component c (the form the library takes maps in)
  std::vector<float> floats(unsigned int c = 0) const {
    const std::vector<double>& v = values();
    const size_t n = cells();
    std::vector<float> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = float(v[c * n + i]);
    return out;
  }
};

class AbstractDataWithGhostNodes : public AbstractData {
 public:
  using AbstractData::AbstractData;
};
class DataWithGhostNodesACLData : public AbstractDataWithGhostNodes {
 public:
  using AbstractDataWithGhostNodes::AbstractDataWithGhostNodes;
};
class DataWithGhostNodesACL : public DataWithGhostNodesACLData {
 public:
  using DataWithGhostNodesACLData::DataWithGhostNodesACLData;
};
typedef std::shared_ptr<AbstractData> SPAbstractData;
typedef std::shared_ptr<AbstractDataWithGhostNodes> SPAbstractDataWithGhostNodes;
typedef std::shared_ptr<DataWithGhostNodesACLData> SPDataWithGhostNodesACLData;
typedef std::shared_ptr<DataWithGhostNodesACL> SPDataWithGhostNodesACL;

template <typename T>
inline SPDataWithGhostNodesACLData generateDataContainerACL_SP(const Block& b, unsigned int n = 1,
                                                               unsigned int gN = 1) {
  return std::make_shared<DataWithGhostNodesACLData>(b, n, gN, acl::typeToTypeID<T>());
}

}  // namespace asl

inline unsigned int acl::VectorOfElements::size() const {
  return data ? data->getEContainerSize() : (unsigned int)constants.size();
}

namespace asl {

// ---- distance functions (src/math/aslDistanceFunction.{h,cxx}:58-165,
//      src/aslGeomInc.cxx:78-210) ------------------------------------------------
//
// Signed distance, negative inside a solid. Evaluated in the container's
// element type (FP32 for float maps), as ASL's generated kernels do.

class DistanceFunction {
 public:
  virtual ~DistanceFunction() {}
  virtual float getDistance(float x, float y, float z) const = 0;
  virtual double getDistance(double x, double y, double z) const = 0;
};
typedef std::shared_ptr<DistanceFunction> SPDistanceFunction;

namespace aslb_detail {
template <class T>
struct V3 {
  T x, y, z;
};
template <class F>
class DFLambda : public DistanceFunction {
  F f_;

 public:
  explicit DFLambda(F f) : f_(f) {}
  float getDistance(float x, float y, float z) const override { return f_(x, y, z); }
  double getDistance(double x, double y, double z) const override { return f_(x, y, z); }
};
template <class F>
inline SPDistanceFunction make_df(F f) {
  return std::make_shared<DFLambda<F>>(f);
}
inline AVec<> unit(const AVec<>& a) {
  const double n = std::sqrt(a * a);
  return a / n;
}
}  // namespace aslb_detail

// |p - c| - R
inline SPDistanceFunction generateDFSphere(double R, const AVec<>& c) {
  const double c0 = c[0], c1 = c[1], c2 = c[2];
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    using T = decltype(x);
    const T d0 = x - T(c0), d1 = y - T(c1), d2 = z - T(c2);
    return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) - T(R);
  });
}

// infinite cylinder of radius R along l through c: |(p - c) - ((p - c).l) l| - R
inline SPDistanceFunction generateDFCylinderInf(double R, const AVec<>& l, const AVec<>& c) {
  const AVec<> u = aslb_detail::unit(l);
  const double u0 = u[0], u1 = u[1], u2 = u[2], c0 = c[0], c1 = c[1], c2 = c[2];
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    using T = decltype(x);
    const T d0 = x - T(c0), d1 = y - T(c1), d2 = z - T(c2);
    const T pr = d0 * T(u0) + d1 * T(u1) + d2 * T(u2);
    const T v0 = d0 - pr * T(u0), v1 = d1 - pr * T(u1), v2 = d2 - pr * T(u2);
    return std::sqrt(v0 * v0 + v1 * v1 + v2 * v2) - T(R);
  });
}

// half space below the plane through p0 with outward normal n: p.n - p0.n
inline SPDistanceFunction generateDFPlane(const AVec<>& n, const AVec<>& p0) {
  const AVec<> u = aslb_detail::unit(n);
  const double u0 = u[0], u1 = u[1], u2 = u[2], b = p0 * u;
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    using T = decltype(x);
    return x * T(u0) + y * T(u1) + z * T(u2) - T(b);
  });
}

// union (min), intersection (max), inversion (negation)
// An operand that is not initialised (a null pointer) leaves the other one
// as the result, as in src/aslGeomInc.cxx:39-66 (programs start unions from
// an empty SPDistanceFunction); both null, or a null negated, is an error.
inline SPDistanceFunction operator|(SPDistanceFunction a, SPDistanceFunction b) {
  if (!a && !b) errorMessage("DistanceFunction::operator| - both operands are not initialized");
  if (!a) return b;
  if (!b) return a;
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    return std::min(a->getDistance(x, y, z), b->getDistance(x, y, z));
  });
}
inline SPDistanceFunction operator&(SPDistanceFunction a, SPDistanceFunction b) {
  if (!a && !b) errorMessage("DistanceFunction::operator& - both operands are not initialized");
  if (!a) return b;
  if (!b) return a;
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    return std::max(a->getDistance(x, y, z), b->getDistance(x, y, z));
  });
}
inline SPDistanceFunction operator-(SPDistanceFunction a) {
  if (!a) errorMessage("DistanceFunction::operator- - operand is not initialized");
  return aslb_detail::make_df([=](auto x, auto y, auto z) { return -a->getDistance(x, y, z); });
}

// finite cylinder: axis vector l (its length is the height) centred at c
inline SPDistanceFunction generateDFCylinder(double R, const AVec<>& l, const AVec<>& c) {
  return generateDFCylinderInf(R, l, c) & generateDFPlane(l, c + l * 0.5) & generateDFPlane(-l, c - l * 0.5);
}

// Convex solids over a convex polygon given by its points in order
// (src/aslGeomInc.cxx:123-160): the intersection of the half-spaces behind
// the plane through each edge, that plane parallel to the polygon's axis (a
// prism, unbounded along the axis) or through the apex a (a pyramid, closed
// by the polygon's own plane).
namespace aslb_detail {
inline AVec<> polygon_center(const std::vector<AVec<double>>& points) {
  if (points.size() < 3) errorMessage("generateDFConvexPolygon: three points at least");
  AVec<> c = points[0];
  for (size_t i = 1; i < points.size(); ++i) c += points[i];
  return c / double(points.size());
}
}  // namespace aslb_detail
inline SPDistanceFunction generateDFConvexPolygonPrism(std::vector<AVec<double>> points) {
  const AVec<> c = aslb_detail::polygon_center(points);
  const AVec<> axis = crossProduct(points[0] - c, points[1] - c);
  SPDistanceFunction res;
  for (size_t i = 0; i < points.size(); ++i) {
    const AVec<>& p = points[i];
    SPDistanceFunction side = generateDFPlane(crossProduct(points[(i + 1) % points.size()] - p, axis), p);
    res = i == 0 ? side : (res & side);
  }
  return res;
}
inline SPDistanceFunction generateDFConvexPolygonPyramid(std::vector<AVec<double>> points, AVec<double> a) {
  const AVec<> c = aslb_detail::polygon_center(points);
  const AVec<> axis = crossProduct(points[0] - c, points[1] - c);
  SPDistanceFunction res = generateDFPlane(-axis, c);
  for (size_t i = 0; i < points.size(); ++i) {
    const AVec<>& p = points[i];
    res = res & generateDFPlane(crossProduct(points[(i + 1) % points.size()] - p, a - p), p);
  }
  return res;
}

// The block's outer layer as a solid: the union of the six half-spaces
// beyond the planes nG - 1/2 cells inside its faces (src/aslGeomInc.cxx:
// 162-183), positive inside those planes and negative beyond them.
inline SPDistanceFunction generateDFInBlock(const Block& b, unsigned int nG) {
  if (nD(b) != 3) errorMessage("generateDFInBlock: three-dimensional blocks only");
  const AVec<> offs(3, (double(nG) - .5) * b.dx);
  const AVec<> p0 = b.position + offs, pE = b.getBPosition() - offs;
  SPDistanceFunction res;
  for (int d = 0; d < 3; ++d) {
    AVec<> nc(3, 0.);
    nc[d] = 1.;
    SPDistanceFunction pair = generateDFPlane(nc, p0) | generateDFPlane(-nc, pE);
    res = d == 0 ? pair : (res | pair);
  }
  return res;
}

// normalize(df, dx) = clip(df / (1.8 dx), -1, 1) (DistFNormalization,
// src/math/aslDistanceFunction.cxx:142-165)
inline SPDistanceFunction normalize(SPDistanceFunction a, double dx) {
  if (!a) errorMessage("DistanceFunction::normalize - argument is not initialized");
  const double factor = 1.0 / dx / 1.8;
  return aslb_detail::make_df([=](auto x, auto y, auto z) {
    using T = decltype(x);
    T d = T(factor) * a->getDistance(x, y, z);
    d = d > T(1) ? T(1) : d;
    return d < T(-1) ? T(-1) : d;
  });
}

// Values of df at the positions of the container's (ghosted) cells,
// position + (i - ghost) dx (src/aslGeomInc.cxx:198-210).
inline void initData(SPAbstractData d, SPDistanceFunction df) {
  if (!df) errorMessage("initData: the distance function is not initialized");
  const Block g = d->getBlock();
  const AVec<int> s = g.getSize();
  std::vector<double>& v = d->values();
  const bool single = d->getTypeID() == acl::TYPE_FLOAT;
  const int gh = (int)d->getGhostLayer();
  const Block& in = d->getInternalBlock();
  size_t k = 0;
  for (int i = 0; i < s[0]; ++i)
    for (int j = 0; j < s[1]; ++j)
      for (int l = 0; l < s[2]; ++l, ++k) {
        if (single) {
          const float x = float(in.position[0]) + (float(i) - float(gh)) * float(in.dx);
          const float y = float(in.position[1]) + (float(j) - float(gh)) * float(in.dx);
          const float z = float(in.position[2]) + (float(l) - float(gh)) * float(in.dx);
          v[k] = df->getDistance(x, y, z);
        } else {
          const double x = in.position[0] + (i - gh) * in.dx;
          const double y = in.position[1] + (j - gh) * in.dx;
          const double z = in.position[2] + (l - gh) * in.dx;
          v[k] = df->getDistance(x, y, z);
        }
      }
}
template <class D>
inline void initData(std::shared_ptr<D> d, SPDistanceFunction df) {
  initData(std::static_pointer_cast<AbstractData>(d), df);
}
// The same value in every cell, per component (src/aslDataInc.h:36-37),
// for host containers.
inline void initData(SPAbstractData d, const AVec<double>& a) {
  if (d->bound()) errorMessage("initData: the container is a view of a device field");
  if (a.getSize() != d->getEContainerSize()) errorMessage("initData: the value has another number of components");
  std::vector<double>& v = d->values();
  const size_t n = d->cells();
  for (unsigned int c = 0; c < a.getSize(); ++c)
    std::fill(v.begin() + (std::ptrdiff_t)(c * n), v.begin() + (std::ptrdiff_t)((c + 1) * n), a[c]);
}
inline void initData(SPAbstractData d, double a) { initData(d, AVec<double>(d->getEContainerSize(), a)); }
template <class D>
inline void initData(std::shared_ptr<D> d, const AVec<double>& a) {
  initData(std::static_pointer_cast<AbstractData>(d), a);
}
template <class D>
inline void initData(std::shared_ptr<D> d, double a) {
  initData(std::static_pointer_cast<AbstractData>(d), a);
}

// A container holding the function's values (ASL's formula-backed data,
// src/aslGenerators.cxx): evaluated once, here.
inline SPAbstractDataWithGhostNodes generateDataContainer_SP(const Block& b, SPDistanceFunction df,
                                                             unsigned int gN, acl::TypeID t) {
  auto d = std::make_shared<DataWithGhostNodesACLData>(b, 1, gN, t);
  initData(std::static_pointer_cast<AbstractData>(d), df);
  return d;
}

// ---- position functions (src/math/aslPositionFunction.h) -----------------------

class PositionFunction {
 public:
  bool rotation = false;
  AVec<> value = AVec<>(3, 0.);   // constant velocity
  AVec<> omega = AVec<>(3, 0.);   // rotation field omega x (r - center)
  AVec<> center = AVec<>(3, 0.);
};
typedef std::shared_ptr<PositionFunction> SPPositionFunction;

inline SPPositionFunction generatePFConstant(const AVec<>& a) {
  auto p = std::make_shared<PositionFunction>();
  p->value = a;
  return p;
}
inline SPPositionFunction generatePFRotationField(const AVec<>& axis, const AVec<>& c) {
  auto p = std::make_shared<PositionFunction>();
  p->rotation = true;
  p->omega = axis;
  p->center = c;
  return p;
}

// ---- numerical methods (src/num/aslNumMethod.h:34-77) -----------------------

class NumMethod {
 public:
  virtual ~NumMethod() {}
  virtual void init() = 0;
  virtual void execute() = 0;
};
typedef std::shared_ptr<NumMethod> SPNumMethod;

class SingleKernelNM : public NumMethod {};

class BCond : public NumMethod {};
typedef std::shared_ptr<BCond> SPBCond;

template <class T> inline void initAll(std::vector<T>& v) {
  for (auto& m : v) m->init();
}
template <class T> inline void executeAll(std::vector<T>& v) {
  for (auto& m : v) m->execute();
}

// src/num/aslBCond.h:309
enum SlicesNames { X0, XE, Y0, YE, Z0, ZE };

// ---- LBGK (src/num/aslLBGK.h:77-171) ------------------------------------------

class LBGK : public SingleKernelNM {
 public:
  typedef SPDataWithGhostNodesACL Data;
  typedef SPDataWithGhostNodesACLData DataD;
  typedef acl::VectorOfElements Param;
  const VectorTemplate* vectorTemplate;

 protected:
  Block block_;
  Param viscosity_;
  int storage_;
  unsigned flags_ = 0;
  bool compVel_, compRho_, compressible_ = true;
  aslb_lbgk* h_ = nullptr;
  DataD rho_, v_;
  Data f_;
  int closure_ = ASLB_CLOSURE_NONE;
  double cs_ = 0.17;
  std::vector<double> g_{0, 0, 0}, om_{0, 0, 0};
  bool hasForce_ = false, hasOmega_ = false;

  static int storage_of(const Param& nu) {
    if (!nu.isConstant()) errorMessage("LBGK: the viscosity must be a constant");
    return nu.type == acl::TYPE_DOUBLE ? ASLB_F64 : ASLB_F32;
  }
  void bind_outputs() {
    const acl::TypeID t = storage_ == ASLB_F64 ? acl::TYPE_DOUBLE : acl::TYPE_FLOAT;
    if (!rho_) rho_ = std::make_shared<DataWithGhostNodesACLData>(block_, 1, 1, t);
    if (!v_) v_ = std::make_shared<DataWithGhostNodesACLData>(block_, 3, 1, t);
    if (!f_) f_ = std::make_shared<DataWithGhostNodesACL>(block_, (unsigned int)vectorTemplate->q, 1, t);
    auto reader = [this](int field) {
      return [this, field](std::vector<double>& out) {
        if (!h_) return;
        aslb_detail::check(aslb_lbgk_read(h_, field, ASLB_F64, out.data()), "LBGK: reading a field back");
      };
    };
    rho_->bind(reader(ASLB_FIELD_RHO));
    v_->bind(reader(ASLB_FIELD_VELOCITY));
    f_->bind(reader(ASLB_FIELD_F));
  }

 public:
  LBGK(Block b, Param nu, const VectorTemplate* vT, bool compVel = true, bool compRho = true)
      : vectorTemplate(vT), block_(b), viscosity_(nu), storage_(storage_of(nu)), compVel_(compVel),
        compRho_(compRho) {
    bind_outputs();
  }
  // the velocity is written into the caller's container v
  LBGK(DataD v, Param nu, const VectorTemplate* vT)
      : vectorTemplate(vT), block_(v->getInternalBlock()), viscosity_(nu), storage_(storage_of(nu)),
        compVel_(true), compRho_(true), v_(v) {
    if (v->getEContainerSize() != 3) errorMessage("LBGK: the velocity container needs 3 components");
    bind_outputs();
  }
  LBGK(const LBGK&) = delete;
  LBGK& operator=(const LBGK&) = delete;
  virtual ~LBGK() {
    if (h_) aslb_lbgk_destroy(h_);
  }

  // The library's domain, created at the first call that needs it
  // (extension: the settings below must come before that).
  aslb_lbgk* handle() {
    if (h_) return h_;
    const AVec<int> s = block_.getSize();
    if (nD(block_) != 3) errorMessage("LBGK: the block must be three-dimensional");
    unsigned fl = flags_;
    if (!compVel_) fl |= ASLB_NO_VELOCITY;
    if (!compRho_) fl |= ASLB_NO_RHO;
    if (!compressible_) fl |= ASLB_INCOMPRESSIBLE;
    aslb_detail::check(aslb_lbgk_create(s[0], s[1], s[2], vectorTemplate->q, storage_, viscosity_.value(), fl, &h_),
                       "LBGK");
    const double pos[3] = {block_.position[0], block_.position[1], block_.position[2]};
    aslb_detail::check(aslb_lbgk_set_position(h_, pos, block_.dx), "LBGK");
    if (closure_ != ASLB_CLOSURE_NONE) aslb_detail::check(aslb_lbgk_set_closure(h_, closure_, cs_), "LBGK");
    if (hasForce_) aslb_detail::check(aslb_lbgk_set_body_force(h_, g_.data()), "LBGK");
    if (hasOmega_) aslb_detail::check(aslb_lbgk_set_omega(h_, om_.data()), "LBGK::setOmega");
    return h_;
  }
  const Block& getBlock() const { return block_; }

  void init() override { handle(); }
  void execute() override { aslb_detail::check(aslb_lbgk_step(handle(), 1), "LBGK::execute"); }

  void setViscosity(Param nu) {
    viscosity_ = nu;
    if (h_) aslb_detail::check(aslb_lbgk_set_viscosity(h_, nu.value()), "LBGK::setViscosity");
  }
  double getViscosity(unsigned int = 0) { return h_ ? aslb_lbgk_get_viscosity(h_) : viscosity_.value(); }
  // angular velocity of the rotating frame (Coriolis term)
  void setOmega(Param w) {
    if (w.size() != 3) errorMessage("LBGK::setOmega: omega needs 3 components");
    om_ = {w.value(0), w.value(1), w.value(2)};
    hasOmega_ = true;
    if (h_) aslb_detail::check(aslb_lbgk_set_omega(h_, om_.data()), "LBGK::setOmega");
  }
  void setVectorTemplate(const VectorTemplate* vT) {
    if (h_) errorMessage("LBGK::setVectorTemplate: the populations already exist");
    vectorTemplate = vT;
    f_.reset();
    bind_outputs();
  }
  const VectorTemplate* getVectorTemplate() const { return vectorTemplate; }
  Data getF() { return f_; }
  DataD getRho() { return rho_; }
  DataD getVelocity() { return v_; }
  void setCompressible(bool flag = true) {
    compressible_ = flag;
    if (h_) aslb_detail::check(aslb_lbgk_set_compressible(h_, flag ? 1 : 0), "LBGK::setCompressible");
  }
  const bool& getCompressible() const { return compressible_; }

  // ---- extensions (no ASL counterpart) ----
  // periodic axes (before the domain exists)
  void setPeriodic(bool x, bool y, bool z) {
    if (h_) errorMessage("LBGK::setPeriodic: the domain already exists");
    flags_ = (flags_ & ~(unsigned)(ASLB_PERIODIC_X | ASLB_PERIODIC_Y | ASLB_PERIODIC_Z)) |
             (x ? ASLB_PERIODIC_X : 0u) | (y ? ASLB_PERIODIC_Y : 0u) | (z ? ASLB_PERIODIC_Z : 0u);
  }
  // body force per unit mass (Guo forcing)
  void setBodyForce(const AVec<>& g) {
    g_ = {g[0], g[1], g[2]};
    hasForce_ = true;
    if (h_) aslb_detail::check(aslb_lbgk_set_body_force(h_, g_.data()), "LBGK::setBodyForce");
  }
  // FP16 shifted storage of the populations, FP32 arithmetic
  void setHalfPrecisionStorage() {
    if (h_) errorMessage("LBGK::setHalfPrecisionStorage: the domain already exists");
    storage_ = ASLB_F16;
  }
  // closure: ASLB_CLOSURE_* and the Smagorinsky constant
  void setClosure(int closure, double cs = 0.17) {
    closure_ = closure;
    cs_ = cs;
    if (h_) aslb_detail::check(aslb_lbgk_set_closure(h_, closure, cs), "LBGK::setClosure");
  }
};
typedef std::shared_ptr<LBGK> SPLBGK;

// LBGKTurbulence's limiter, evaluated on a defined f_eq (the reference reads
// f_eq before assigning it, src/num/aslLBGK.cxx:315-352).
class LBGKTurbulence : public LBGK {
 public:
  LBGKTurbulence(DataD v, Param nu, const VectorTemplate* vT) : LBGK(v, nu, vT) { closure_ = ASLB_CLOSURE_ASL_INTENT; }
  LBGKTurbulence(Block b, Param nu, const VectorTemplate* vT, bool compVel = true, bool compRho = true)
      : LBGK(b, nu, vT, compVel, compRho) {
    closure_ = ASLB_CLOSURE_ASL_INTENT;
  }
};
typedef std::shared_ptr<LBGKTurbulence> SPLBGKTurbulence;

// src/num/aslLBGK.h:137-159 (computeRho / computeVelocity / computeRhoVelocity
// are declared there and never defined; here they compute the fields from the
// populations as they stand).
class LBGKUtilities {
  SPLBGK num;

  static std::vector<double> field(const acl::VectorOfElements& p, unsigned int ncomp, size_t cells) {
    std::vector<double> out((size_t)ncomp * cells);
    if (p.isConstant()) {
      if (p.size() != ncomp) errorMessage("LBGKUtilities::initF: wrong number of components");
      for (unsigned int c = 0; c < ncomp; ++c) std::fill(out.begin() + c * cells, out.begin() + (c + 1) * cells, p.value(c));
    } else {
      if (p.data->getEContainerSize() != ncomp || p.data->cells() != cells)
        errorMessage("LBGKUtilities::initF: the field does not match the domain");
      out = p.data->values();
    }
    return out;
  }

 public:
  explicit LBGKUtilities(SPLBGK lbgk) : num(lbgk) {}
  void computeRho() { aslb_detail::check(aslb_lbgk_compute_macro(num->handle(), 1, 0), "LBGKUtilities::computeRho"); }
  void computeVelocity() {
    aslb_detail::check(aslb_lbgk_compute_macro(num->handle(), 0, 1), "LBGKUtilities::computeVelocity");
  }
  void computeRhoVelocity() {
    aslb_detail::check(aslb_lbgk_compute_macro(num->handle(), 1, 1), "LBGKUtilities::computeRhoVelocity");
  }
  void initF(acl::VectorOfElements rho, acl::VectorOfElements vel) {
    aslb_lbgk* h = num->handle();
    if (rho.isConstant() && vel.isConstant()) {
      if (vel.size() != 3) errorMessage("LBGKUtilities::initF: the velocity needs 3 components");
      const double u[3] = {vel.value(0), vel.value(1), vel.value(2)};
      aslb_detail::check(aslb_lbgk_init_f(h, rho.value(), u), "LBGKUtilities::initF");
      return;
    }
    const size_t n = offset(num->getBlock(), 1).getSize()[0] * (size_t)offset(num->getBlock(), 1).getSize()[1] *
                     offset(num->getBlock(), 1).getSize()[2];
    const std::vector<double> r = field(rho, 1, n), u = field(vel, 3, n);
    aslb_detail::check(aslb_lbgk_init_f_fields(h, r.data(), u.data()), "LBGKUtilities::initF");
  }
  // the density is supposed to be 1
  void initF(acl::VectorOfElements vel) { initF(acl::generateVEConstant(1.0), vel); }
};
typedef std::shared_ptr<LBGKUtilities> SPLBGKUtilities;

}  // namespace asl

#include "aslb_asl_bc.hpp"

#endif  // ASLB_ASL_HPP
