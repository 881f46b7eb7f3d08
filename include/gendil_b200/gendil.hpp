// gendil_b200/gendil.hpp -- C++20 host facade with GenDiL's names over the dgop C ABI.
//
// A GenDiL program on the mass / upwind-advection path compiles against this header with its
// `using namespace gendil;` replaced by `using namespace gendil_b200;` (or a namespace alias):
// meshes, finite elements, spaces, integration rules, Vector, FillRandom, the operator factories
// (MakeMassFiniteElementOperator, MakeAdvectionOperator, MakeMassAdvectionOperator), the weak-form
// DSL (TrialSpace / TestSpace, Cells / InteriorFacets / BoundaryFacets, integrate, grad, dot, jump,
// upwind, Normal, MakeCoefficient, MakeVectorCoefficient, MakeWeakFormContext,
// MakeGenericOperator) and the Krylov drivers (ConjugateGradient, GMRES_no_alloc) keep the
// reference's call shapes (include/gendil/gendil.hpp of the reference).  Every operator runs on
// the sm_100a kernels behind libdgop.so; there is no host execution path.
//
// Weak forms are recognised, not interpreted: the hot-path forms
//   integrate(cells, [c *] u * v)                                  mass (massoperator.hpp:65-83)
//   integrate(cells, -u * dot(beta, grad(v)))                      cell advection (advectionoperator.hpp:293-331)
//   integrate(interior_facets, upwind(beta, u) * jump(v))          interior upwind flux (upwind.hpp:43-76)
//   integrate(boundary_facets, [c *] dot(beta, Normal{}) * u * v)  outflow boundary flux, c the outflow
//                                                                  indicator (checked on every boundary point)
// in the combinations {mass}, {cell, interior}, {cell, interior, boundary},
// {mass, cell, interior}, {mass, cell, interior, boundary} map to one fused kernel; anything else
// throws gendil_b200::Error naming the unsupported term.
//
// Coefficients are functions of the physical coordinate X.  The kernels take each scalar
// coefficient as constant + sum_t prod_k T_tk(X_k) over the per-axis sample coordinates; the
// facade finds that form by probing the function on the mesh's coordinate lines (additive blocks
// of interacting axes, each block a constant plus a product of 1D functions) and verifies it on
// every sample point of the tensor grid (on 2^20 pseudo-random points when the grid has more than
// 2^22).  A function outside that class is rejected with an error.
#pragma once

#include <cuda_runtime.h>
#include <dgop.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace gendil_b200 {

using Real = double;
using Integer = std::size_t;
using GlobalIndex = std::size_t;

class Error : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

namespace detail {

inline void check(int rc, const std::string& what) {
  if (rc != DGOP_OK) throw Error(what + ": " + dgop_last_error());
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(std::string(what) + ": " + cudaGetErrorString(e));
}

// String literal as a template argument (TrialSpace<"u">, Cells<"mesh">, ...).
template <std::size_t N>
struct FixedString {
  char s[N]{};
  constexpr FixedString(const char (&v)[N]) {
    for (std::size_t i = 0; i < N; ++i) s[i] = v[i];
  }
  std::string str() const { return std::string(s); }
};

}  // namespace detail

// ------------------------------------------------------------------------- kernel policies
// Accepted for source compatibility; every facade operator runs the sm_100a kernels.
struct SerialKernelConfiguration {};
template <Integer... Sizes>
struct ThreadBlockLayout {};
template <typename Layout, auto... Rest>
struct ThreadFirstKernelConfiguration {};
using DeviceKernelConfiguration = ThreadFirstKernelConfiguration<ThreadBlockLayout<>>;

// ------------------------------------------------------------------------- mesh, element, space
// CartesianMesh<Dim> (Meshes/MeshDataStructures/CartesianMesh/cartesianndmesh.hpp:44-80)
template <Integer Dim>
struct CartesianMesh {
  static_assert(Dim >= 1 && Dim <= 6, "dimensions 1..6");
  std::array<GlobalIndex, Dim> sizes;
  std::array<Real, Dim> h;
  std::array<Real, Dim> mesh_origin;
  std::array<int, Dim> is_periodic_boundary{};

  CartesianMesh(const std::array<GlobalIndex, Dim>& sizes, const std::array<Real, Dim>& h,
                const std::array<Real, Dim>& origin)
      : sizes(sizes), h(h), mesh_origin(origin) {}
  CartesianMesh(const std::array<GlobalIndex, Dim>& sizes, const std::array<Real, Dim>& h,
                const std::array<Real, Dim>& origin, bool periodic)
      : sizes(sizes), h(h), mesh_origin(origin) {
    is_periodic_boundary.fill(periodic ? 1 : 0);
  }
  CartesianMesh(const std::array<GlobalIndex, Dim>& sizes, const std::array<Real, Dim>& h,
                const std::array<Real, Dim>& origin, const std::array<int, Dim>& periodic)
      : sizes(sizes), h(h), mesh_origin(origin), is_periodic_boundary(periodic) {}

  Integer GetNumberOfCells() const {
    Integer n = 1;
    for (auto s : sizes) n *= s;
    return n;
  }
  GlobalIndex Size(GlobalIndex i) const { return sizes[i]; }
};

template <Integer... Orders>
struct FiniteElementOrders {};

template <Integer Dim>
struct FiniteElement {
  int order;
  int basis;  // DGOP_BASIS_GLL or DGOP_BASIS_GL
};

// MakeLobattoFiniteElement / MakeLegendreFiniteElement (finiteelement.hpp:103,109)
template <Integer O0, Integer... Os>
FiniteElement<1 + sizeof...(Os)> MakeLobattoFiniteElement(FiniteElementOrders<O0, Os...>) {
  static_assert(((Os == O0) && ...), "the kernels take the same order on every axis");
  static_assert(O0 <= 7, "orders 0..7");
  return {int(O0), DGOP_BASIS_GLL};
}
template <Integer O0, Integer... Os>
FiniteElement<1 + sizeof...(Os)> MakeLegendreFiniteElement(FiniteElementOrders<O0, Os...>) {
  static_assert(((Os == O0) && ...), "the kernels take the same order on every axis");
  static_assert(O0 <= 7, "orders 0..7");
  return {int(O0), DGOP_BASIS_GL};
}

// FiniteElementSpace (finiteelementspace.hpp:84): an L2 space on a Cartesian mesh.
template <Integer D>
class FiniteElementSpace {
 public:
  static constexpr Integer dim = D;
  FiniteElementSpace(const CartesianMesh<D>& mesh, const FiniteElement<D>& fe) : mesh_(mesh), fe_(fe) {
    int64_t n[D];
    for (Integer k = 0; k < D; ++k) n[k] = (int64_t)mesh.sizes[k];
    dgop_space* sp = nullptr;
    detail::check(dgop_space_create((int)D, n, mesh.h.data(), mesh.mesh_origin.data(),
                                    mesh.is_periodic_boundary.data(), fe.order, fe.basis, &sp),
                  "MakeFiniteElementSpace");
    space_ = std::shared_ptr<dgop_space>(sp, [](dgop_space* s) { dgop_space_destroy(s); });
  }
  Integer GetNumberOfFiniteElementDofs() const { return (Integer)dgop_space_num_dofs(space_.get()); }
  Integer GetNumberOfFiniteElements() const { return (Integer)dgop_space_num_elements(space_.get()); }
  const CartesianMesh<D>& GetMesh() const { return mesh_; }
  const FiniteElement<D>& GetFiniteElement() const { return fe_; }
  const dgop_space* handle() const { return space_.get(); }

 private:
  CartesianMesh<D> mesh_;
  FiniteElement<D> fe_;
  std::shared_ptr<dgop_space> space_;
};

template <Integer D>
FiniteElementSpace<D> MakeFiniteElementSpace(const CartesianMesh<D>& mesh, const FiniteElement<D>& fe) {
  return FiniteElementSpace<D>(mesh, fe);
}

template <Integer... Q>
struct IntegrationRuleNumPoints {};

template <Integer D>
struct IntegrationRule {
  int q;  // Gauss-Legendre points per axis
};

// MakeIntegrationRule (integrationrule.hpp): tensor Gauss-Legendre, same count on every axis.
template <Integer Q0, Integer... Qs>
IntegrationRule<1 + sizeof...(Qs)> MakeIntegrationRule(IntegrationRuleNumPoints<Q0, Qs...>) {
  static_assert(((Qs == Q0) && ...), "the kernels take the same number of points on every axis");
  static_assert(Q0 >= 1 && Q0 <= 8, "1..8 points per axis");
  return {int(Q0)};
}

// ------------------------------------------------------------------------- Vector
// Host/device mirrored vector with validity flags (Algebra/vector.hpp:84-160).
class Vector {
 public:
  Vector() = default;
  explicit Vector(Integer n) : n_(n) {}
  explicit Vector(int n) : n_((Integer)n) {}
  template <Integer D>
  explicit Vector(const FiniteElementSpace<D>& fes) : n_(fes.GetNumberOfFiniteElementDofs()) {}
  Vector(const Vector& o) : n_(o.n_) { copy_from(o); }
  Vector(Vector&& o) noexcept { swap(o); }
  Vector& operator=(const Vector& o) {
    if (this != &o) {
      if (n_ != o.n_) {
        release();
        n_ = o.n_;
      }
      copy_from(o);
    }
    return *this;
  }
  Vector& operator=(Vector&& o) noexcept {
    if (this != &o) {
      release();
      swap(o);
    }
    return *this;
  }
  ~Vector() { release(); }

  Integer Size() const { return n_; }

  const Real* ReadHostData() const {
    sync_host();
    return host_.get();
  }
  Real* WriteHostData() {
    alloc_host();
    host_valid_ = true;
    dev_valid_ = false;
    return host_.get();
  }
  Real* ReadWriteHostData() {
    sync_host();
    dev_valid_ = false;
    return host_.get();
  }
  const Real* ReadDeviceData() const {
    sync_dev();
    return dev_;
  }
  Real* WriteDeviceData() {
    alloc_dev();
    dev_valid_ = true;
    host_valid_ = false;
    return dev_;
  }
  Real* ReadWriteDeviceData() {
    sync_dev();
    host_valid_ = false;
    return dev_;
  }

  Real& operator[](Integer i) { return ReadWriteHostData()[i]; }
  const Real& operator[](Integer i) const { return ReadHostData()[i]; }

  Vector& operator=(Real v) {
    Real* p = WriteHostData();
    std::fill(p, p + n_, v);
    return *this;
  }
  Vector& operator+=(const Vector& o) { return zip(o, [](Real& a, Real b) { a = a + b; }); }
  Vector& operator-=(const Vector& o) { return zip(o, [](Real& a, Real b) { a = a - b; }); }
  Vector& operator*=(Real s) {
    Real* p = ReadWriteHostData();
    for (Integer i = 0; i < n_; ++i) p[i] *= s;
    return *this;
  }
  Vector& operator/=(Real s) {
    Real* p = ReadWriteHostData();
    for (Integer i = 0; i < n_; ++i) p[i] /= s;
    return *this;
  }

 private:
  Integer n_ = 0;
  mutable std::unique_ptr<Real[]> host_;
  mutable Real* dev_ = nullptr;
  mutable bool host_valid_ = false, dev_valid_ = false;

  void alloc_host() const {
    if (!host_ && n_) host_.reset(new Real[n_]);
  }
  void alloc_dev() const {
    if (!dev_ && n_) detail::cuda_check(cudaMalloc(&dev_, n_ * sizeof(Real)), "Vector: cudaMalloc");
  }
  void sync_host() const {
    alloc_host();
    if (!host_valid_ && dev_valid_ && n_)
      detail::cuda_check(cudaMemcpy(host_.get(), dev_, n_ * sizeof(Real), cudaMemcpyDeviceToHost),
                         "Vector: device to host copy");
    host_valid_ = true;
  }
  void sync_dev() const {
    alloc_dev();
    if (!dev_valid_ && host_valid_ && n_)
      detail::cuda_check(cudaMemcpy(dev_, host_.get(), n_ * sizeof(Real), cudaMemcpyHostToDevice),
                         "Vector: host to device copy");
    dev_valid_ = true;
  }
  void release() {
    if (dev_) cudaFree(dev_);
    dev_ = nullptr;
    host_.reset();
    host_valid_ = dev_valid_ = false;
  }
  void swap(Vector& o) noexcept {
    std::swap(n_, o.n_);
    std::swap(host_, o.host_);
    std::swap(dev_, o.dev_);
    std::swap(host_valid_, o.host_valid_);
    std::swap(dev_valid_, o.dev_valid_);
  }
  void copy_from(const Vector& o) {
    if (!n_) return;
    if (o.dev_valid_) {
      alloc_dev();
      detail::cuda_check(cudaMemcpy(dev_, o.dev_, n_ * sizeof(Real), cudaMemcpyDeviceToDevice), "Vector copy");
      dev_valid_ = true;
      host_valid_ = false;
    } else if (o.host_valid_) {
      alloc_host();
      std::memcpy(host_.get(), o.host_.get(), n_ * sizeof(Real));
      host_valid_ = true;
      dev_valid_ = false;
    }
  }
  template <typename F>
  Vector& zip(const Vector& o, F f) {
    if (o.n_ != n_) throw Error("Vector sizes do not match");
    Real* p = ReadWriteHostData();
    const Real* q = o.ReadHostData();
    for (Integer i = 0; i < n_; ++i) f(p[i], q[i]);
    return *this;
  }
};

// FillRandom (Algebra/vector.hpp:632-647): std::mt19937(seed), uniform in [min, max), in order.
inline void FillRandom(Vector& v, unsigned int seed = 12345, Real min_value = Real(-1), Real max_value = Real(1)) {
  detail::check(dgop_fill_random(v.WriteHostData(), (int64_t)v.Size(), seed, min_value, max_value), "FillRandom");
}

inline Real Dot(const Vector& a, const Vector& b) {
  if (a.Size() != b.Size()) throw Error("Dot: vector sizes do not match");
  const Real* p = a.ReadHostData();
  const Real* q = b.ReadHostData();
  Real s = 0.0;
  for (Integer i = 0; i < a.Size(); ++i) s += p[i] * q[i];
  return s;
}

// ------------------------------------------------------------------------- coefficient fields
struct PhysicalCoordinate {};

namespace detail {

struct ScalarField {
  std::string name;
  virtual ~ScalarField() = default;
  virtual Real eval(int D, const Real* X) const = 0;
};

struct VectorField {
  std::string name;
  virtual ~VectorField() = default;
  virtual void eval(int D, const Real* X, Real* out) const = 0;
};

template <int D>
std::array<Real, D> to_array(const Real* X) {
  std::array<Real, D> a;
  for (int k = 0; k < D; ++k) a[k] = X[k];
  return a;
}

template <typename Fn>
struct ScalarFieldImpl final : ScalarField {
  Fn fn;
  explicit ScalarFieldImpl(Fn f, std::string n) : fn(std::move(f)) { name = std::move(n); }
  template <int D>
  Real call(const Real* X) const {
    if constexpr (std::is_arithmetic_v<Fn>) {
      return (Real)fn;
    } else if constexpr (std::is_invocable_v<const Fn&, const std::array<Real, D>&>) {
      return (Real)fn(to_array<D>(X));
    } else {
      throw Error("coefficient '" + name + "' cannot be evaluated at a point of dimension " + std::to_string(D));
    }
  }
  Real eval(int D, const Real* X) const override {
    switch (D) {
      case 1: return call<1>(X);
      case 2: return call<2>(X);
      case 3: return call<3>(X);
      case 4: return call<4>(X);
      case 5: return call<5>(X);
      case 6: return call<6>(X);
    }
    throw Error("dimension outside 1..6");
  }
};

// A vector field is either X -> std::array<Real, D> (MakeVectorCoefficient) or the legacy
// advection signature (X, Real (&v)[D]) (advectionoperator.hpp:317).
template <typename Fn>
struct VectorFieldImpl final : VectorField {
  Fn fn;
  explicit VectorFieldImpl(Fn f, std::string n) : fn(std::move(f)) { name = std::move(n); }
  template <int D>
  void call(const Real* X, Real* out) const {
    const auto a = to_array<D>(X);
    if constexpr (std::is_invocable_v<const Fn&, const std::array<Real, D>&, Real(&)[D]>) {
      Real v[D];
      fn(a, v);
      for (int k = 0; k < D; ++k) out[k] = v[k];
    } else if constexpr (std::is_invocable_v<const Fn&, const std::array<Real, D>&>) {
      const auto v = fn(a);
      for (int k = 0; k < D; ++k) out[k] = (Real)v[k];
    } else {
      throw Error("vector coefficient '" + name + "' cannot be evaluated at a point of dimension " +
                  std::to_string(D));
    }
  }
  void eval(int D, const Real* X, Real* out) const override {
    switch (D) {
      case 1: return call<1>(X, out);
      case 2: return call<2>(X, out);
      case 3: return call<3>(X, out);
      case 4: return call<4>(X, out);
      case 5: return call<5>(X, out);
      case 6: return call<6>(X, out);
    }
    throw Error("dimension outside 1..6");
  }
};

template <typename Fn>
std::shared_ptr<const ScalarField> make_scalar(Fn fn, std::string name) {
  return std::make_shared<ScalarFieldImpl<Fn>>(std::move(fn), std::move(name));
}
template <typename Fn>
std::shared_ptr<const VectorField> make_vector(Fn fn, std::string name) {
  return std::make_shared<VectorFieldImpl<Fn>>(std::move(fn), std::move(name));
}

// ---- the per-axis sample grid of an operator and the separated form of a coefficient

// Coordinates of the coefficient samples along each axis: element e, point j < q is Gauss point
// j, j = q the element's lower face, j = q + 1 its upper face (dgop_space_coordinates).
struct Grid {
  int D = 0, q = 0;
  std::vector<int64_t> nelem;
  std::vector<std::vector<Real>> x;  // x[k][e * (q + 2) + j]
  std::vector<int> periodic;
  int64_t m(int k) const { return (int64_t)x[k].size(); }
};

inline Grid make_grid(const dgop_space* sp, int D, const int64_t* nelem, const int* periodic, int q) {
  Grid g;
  g.D = D;
  g.q = q;
  g.x.resize(D);
  for (int k = 0; k < D; ++k) {
    g.nelem.push_back(nelem[k]);
    g.periodic.push_back(periodic ? periodic[k] : 0);
    g.x[k].resize((size_t)nelem[k] * (q + 2));
    check(dgop_space_coordinates(sp, q, k, g.x[k].data()), "coefficient grid");
  }
  return g;
}

// constant + sum_t prod_k T[t][k] (an empty table is the factor 1)
struct Separated {
  Real constant = 0.0;
  std::vector<std::array<std::vector<Real>, 6>> terms;
  void fill(dgop_coef& c) const {
    std::memset(&c, 0, sizeof(c));
    c.constant = constant;
    c.nterms = (int)terms.size();
    for (size_t t = 0; t < terms.size(); ++t)
      for (int k = 0; k < 6; ++k) c.tables[t][k] = terms[t][k].empty() ? nullptr : terms[t][k].data();
  }
  Real eval(const int64_t* idx, int D) const {
    Real s = constant;
    for (const auto& t : terms) {
      Real p = 1.0;
      bool any = false;
      for (int k = 0; k < D; ++k)
        if (!t[k].empty()) {
          p = any ? p * t[k][idx[k]] : t[k][idx[k]];
          any = true;
        }
      s += p;
    }
    return s;
  }
};

class GridFunction {
 public:
  GridFunction(const Grid& g, std::function<Real(const Real*)> f) : g_(g), f_(std::move(f)) {}
  Real operator()(const int64_t* idx) const {
    Real X[6];
    for (int k = 0; k < g_.D; ++k) X[k] = g_.x[k][idx[k]];
    return f_(X);
  }

 private:
  const Grid& g_;
  std::function<Real(const Real*)> f_;
};

// Pseudo-random sample points (a fixed linear congruential sequence) or every point of the grid.
template <typename F>
void for_verification_points(const Grid& g, F&& visit) {
  double total = 1.0;
  for (int k = 0; k < g.D; ++k) total *= (double)g.m(k);
  int64_t idx[6] = {0, 0, 0, 0, 0, 0};
  if (total <= double(1 << 22)) {
    const int64_t n = (int64_t)total;
    for (int64_t i = 0; i < n; ++i) {
      int64_t r = i;
      for (int k = 0; k < g.D; ++k) {
        idx[k] = r % g.m(k);
        r /= g.m(k);
      }
      visit(idx);
    }
    return;
  }
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int i = 0; i < (1 << 20); ++i) {
    for (int k = 0; k < g.D; ++k) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      idx[k] = (int64_t)((s >> 33) % (uint64_t)g.m(k));
    }
    visit(idx);
  }
}

// Finds constant + sum over additive blocks of (c_B + prod_{k in B} g_k(x_k)) for f on the grid.
inline Separated separate(const Grid& g, const std::function<Real(const Real*)>& fx, const std::string& what) {
  const int D = g.D;
  GridFunction f(g, fx);
  int64_t b[6];
  for (int k = 0; k < D; ++k) b[k] = g.m(k) / 2;
  const Real fb = f(b);
  // lines through b
  std::vector<std::vector<Real>> L(D);
  Real scale = std::fabs(fb);
  std::vector<int> dep;
  for (int k = 0; k < D; ++k) {
    int64_t idx[6];
    std::copy(b, b + D, idx);
    L[k].resize(g.m(k));
    bool varies = false;
    for (int64_t t = 0; t < g.m(k); ++t) {
      idx[k] = t;
      L[k][t] = f(idx);
      scale = std::max(scale, std::fabs(L[k][t]));
      varies = varies || L[k][t] != fb;
    }
    if (varies) dep.push_back(k);
  }
  if (!std::isfinite(scale)) throw Error(what + ": the coefficient is not finite on the mesh");
  const Real tol = 1e-14 * std::max(scale, 1e-300);
  // probe indices along each axis (at most 48, always including b)
  auto probes = [&](int k) {
    std::vector<int64_t> p;
    const int64_t m = g.m(k);
    const int64_t step = std::max<int64_t>(1, m / 47);
    for (int64_t t = 0; t < m; t += step) p.push_back(t);
    p.push_back(b[k]);
    return p;
  };
  // interaction graph: axes i, j interact when the mixed difference on their plane is non-zero
  const int nd = (int)dep.size();
  std::vector<int> comp(nd);
  for (int i = 0; i < nd; ++i) comp[i] = i;
  std::function<int(int)> find = [&](int i) { return comp[i] == i ? i : comp[i] = find(comp[i]); };
  for (int a = 0; a < nd; ++a)
    for (int c = a + 1; c < nd; ++c) {
      const int i = dep[a], j = dep[c];
      bool inter = false;
      int64_t idx[6];
      std::copy(b, b + D, idx);
      for (int64_t s : probes(i)) {
        for (int64_t t : probes(j)) {
          idx[i] = s;
          idx[j] = t;
          const Real v = f(idx) - L[i][s] - L[j][t] + fb;
          if (std::fabs(v) > tol) {
            inter = true;
            break;
          }
        }
        if (inter) break;
      }
      if (inter) comp[find(a)] = find(c);
    }
  std::map<int, std::vector<int>> blocks;
  for (int a = 0; a < nd; ++a) blocks[find(a)].push_back(dep[a]);
  if ((int)blocks.size() > DGOP_MAX_TERMS)
    throw Error(what + ": the coefficient needs " + std::to_string(blocks.size()) + " terms (at most " +
                std::to_string(DGOP_MAX_TERMS) + ")");
  Separated sep;
  sep.constant = blocks.empty() ? fb : -(Real)(blocks.size() - 1) * fb;
  for (auto& kv : blocks) {
    const std::vector<int>& B = kv.second;
    std::array<std::vector<Real>, 6> term;
    if (B.size() == 1) {
      term[B[0]] = L[B[0]];
    } else {
      // A(x_B) = f(x_B, b_rest) = c + prod g_k: c from the rank-one condition on the plane of
      // the first two axes, at the probe point where it is best conditioned
      const int i = B[0], j = B[1];
      int64_t idx[6];
      std::copy(b, b + D, idx);
      Real best = 0.0, c = 0.0;
      for (int64_t s : probes(i))
        for (int64_t t : probes(j)) {
          idx[i] = s;
          idx[j] = t;
          const Real A = f(idx);
          const Real den = A + fb - L[i][s] - L[j][t];
          if (std::fabs(den) > best) {
            best = std::fabs(den);
            c = (A * fb - L[i][s] * L[j][t]) / den;
          }
        }
      const Real p0 = fb - c;
      if (best <= tol || std::fabs(p0) <= tol)
        throw Error(what + ": the coefficient is not a sum of products of one-dimensional functions");
      sep.constant += c;
      term[B[0]].resize(L[B[0]].size());
      for (size_t t = 0; t < L[B[0]].size(); ++t) term[B[0]][t] = L[B[0]][t] - c;
      for (size_t u = 1; u < B.size(); ++u) {
        const int k = B[u];
        term[k].resize(L[k].size());
        for (size_t t = 0; t < L[k].size(); ++t) term[k][t] = (L[k][t] - c) / p0;
      }
    }
    sep.terms.push_back(std::move(term));
  }
  Real worst = 0.0;
  for_verification_points(g, [&](const int64_t* idx) {
    worst = std::max(worst, std::fabs(f(idx) - sep.eval(idx, D)));
  });
  if (!(worst <= tol))
    throw Error(what + ": the coefficient is not a sum of products of one-dimensional functions of the "
                       "coordinates (deviation " + std::to_string(worst) + ")");
  return sep;
}

// Calls visit(X, axis, side) at every Gauss point of every boundary face of the mesh.
template <typename F>
void for_boundary_points(const Grid& g, F&& visit) {
  const int D = g.D, q = g.q;
  for (int k = 0; k < D; ++k) {
    if (g.periodic[k]) continue;
    for (int side = 0; side < 2; ++side) {
      const int64_t e = side == 0 ? 0 : g.nelem[k] - 1;
      const Real xk = g.x[k][e * (q + 2) + q + side];
      int64_t cnt = 1;
      for (int a = 0; a < D; ++a)
        if (a != k) cnt *= g.nelem[a] * q;
      for (int64_t i = 0; i < cnt; ++i) {
        Real X[6];
        int64_t r = i;
        for (int a = 0; a < D; ++a) {
          if (a == k) {
            X[a] = xk;
            continue;
          }
          const int64_t m = g.nelem[a] * q;
          const int64_t t = r % m;
          r /= m;
          X[a] = g.x[a][(t / q) * (q + 2) + t % q];
        }
        visit(X, k, side);
      }
    }
  }
}

}  // namespace detail

// MakeCoefficient<"name", PhysicalCoordinate>(fn) / MakeVectorCoefficient (coefficient.hpp:546,554)
template <detail::FixedString Name, typename Tag = PhysicalCoordinate>
struct Coefficient {
  std::shared_ptr<const detail::ScalarField> field;
};
template <detail::FixedString Name, typename Tag = PhysicalCoordinate>
struct VectorCoefficient {
  std::shared_ptr<const detail::VectorField> field;
};

template <detail::FixedString Name, typename Tag, typename Fn>
Coefficient<Name, Tag> MakeCoefficient(const Fn& fn) {
  static_assert(std::is_same_v<Tag, PhysicalCoordinate>, "coefficients are functions of the PhysicalCoordinate");
  return {detail::make_scalar(fn, Name.str())};
}
template <detail::FixedString Name, typename Tag, typename Fn>
VectorCoefficient<Name, Tag> MakeVectorCoefficient(const Fn& fn) {
  static_assert(std::is_same_v<Tag, PhysicalCoordinate>, "coefficients are functions of the PhysicalCoordinate");
  return {detail::make_vector(fn, Name.str())};
}

// ------------------------------------------------------------------------- weak-form DSL
namespace detail {
enum class NK { Trial, Test, Grad, Dot, Mul, Neg, Scalar, Coef, VecCoef, Normal, Jump, Average, Upwind, Add };
struct Node;
using NodeP = std::shared_ptr<const Node>;
struct Node {
  NK k;
  Real value = 0.0;
  std::string name;
  NodeP a, b;
  std::shared_ptr<const ScalarField> sf;
  std::shared_ptr<const VectorField> vf;
};
inline NodeP mk(NK k, NodeP a = {}, NodeP b = {}) {
  auto n = std::make_shared<Node>();
  n->k = k;
  n->a = std::move(a);
  n->b = std::move(b);
  return n;
}
}  // namespace detail

struct Expr {
  detail::NodeP node;
};
struct Normal {};
template <detail::FixedString Name>
struct TrialSpace {};
template <detail::FixedString Name>
struct TestSpace {};

inline Expr to_expr(const Expr& e) { return e; }
inline Expr to_expr(const Normal&) { return {detail::mk(detail::NK::Normal)}; }
template <detail::FixedString Name>
Expr to_expr(const TrialSpace<Name>&) {
  auto n = std::make_shared<detail::Node>();
  n->k = detail::NK::Trial;
  n->name = Name.str();
  return {n};
}
template <detail::FixedString Name>
Expr to_expr(const TestSpace<Name>&) {
  auto n = std::make_shared<detail::Node>();
  n->k = detail::NK::Test;
  n->name = Name.str();
  return {n};
}
template <detail::FixedString Name, typename Tag>
Expr to_expr(const Coefficient<Name, Tag>& c) {
  auto n = std::make_shared<detail::Node>();
  n->k = detail::NK::Coef;
  n->name = Name.str();
  n->sf = c.field;
  return {n};
}
template <detail::FixedString Name, typename Tag>
Expr to_expr(const VectorCoefficient<Name, Tag>& c) {
  auto n = std::make_shared<detail::Node>();
  n->k = detail::NK::VecCoef;
  n->name = Name.str();
  n->vf = c.field;
  return {n};
}

template <typename T>
concept ExprLike = requires(const T& t) {
  { to_expr(t) } -> std::same_as<Expr>;
};

template <ExprLike A, ExprLike B>
Expr operator*(const A& a, const B& b) {
  return {detail::mk(detail::NK::Mul, to_expr(a).node, to_expr(b).node)};
}
template <ExprLike A>
Expr operator*(Real s, const A& a) {
  auto n = std::make_shared<detail::Node>();
  n->k = detail::NK::Scalar;
  n->value = s;
  return {detail::mk(detail::NK::Mul, n, to_expr(a).node)};
}
template <ExprLike A>
Expr operator*(const A& a, Real s) {
  return s * a;
}
template <ExprLike A>
Expr operator-(const A& a) {
  return {detail::mk(detail::NK::Neg, to_expr(a).node)};
}
template <ExprLike A, ExprLike B>
Expr operator+(const A& a, const B& b) {
  return {detail::mk(detail::NK::Add, to_expr(a).node, to_expr(b).node)};
}
template <ExprLike A, ExprLike B>
Expr operator-(const A& a, const B& b) {
  return a + (-b);
}
template <ExprLike A>
Expr grad(const A& a) {
  return {detail::mk(detail::NK::Grad, to_expr(a).node)};
}
template <ExprLike A, ExprLike B>
Expr dot(const A& a, const B& b) {
  return {detail::mk(detail::NK::Dot, to_expr(a).node, to_expr(b).node)};
}
template <ExprLike A>
Expr jump(const A& a) {
  return {detail::mk(detail::NK::Jump, to_expr(a).node)};
}
template <ExprLike A>
Expr average(const A& a) {
  return {detail::mk(detail::NK::Average, to_expr(a).node)};
}
template <ExprLike A, ExprLike B>
Expr upwind(const A& beta, const B& u) {
  return {detail::mk(detail::NK::Upwind, to_expr(beta).node, to_expr(u).node)};
}

enum class DomainKind { Cells, InteriorFacets, BoundaryFacets };
template <detail::FixedString Name>
struct Cells {};
template <detail::FixedString Name>
struct InteriorFacets {};
template <detail::FixedString Name>
struct BoundaryFacets {};

struct Integral {
  DomainKind kind;
  std::string domain;
  detail::NodeP expr;
};
struct WeakForm {
  std::vector<Integral> terms;
};
template <detail::FixedString N, ExprLike E>
WeakForm integrate(const Cells<N>&, const E& e) {
  return {{{DomainKind::Cells, N.str(), to_expr(e).node}}};
}
template <detail::FixedString N, ExprLike E>
WeakForm integrate(const InteriorFacets<N>&, const E& e) {
  return {{{DomainKind::InteriorFacets, N.str(), to_expr(e).node}}};
}
template <detail::FixedString N, ExprLike E>
WeakForm integrate(const BoundaryFacets<N>&, const E& e) {
  return {{{DomainKind::BoundaryFacets, N.str(), to_expr(e).node}}};
}
inline WeakForm operator+(WeakForm a, const WeakForm& b) {
  a.terms.insert(a.terms.end(), b.terms.begin(), b.terms.end());
  return a;
}

// MakeWeakFormContext(MakeTrialField<"u">(fes), MakeIntegrationDomain<"mesh">(fes))
// (weakformcontext.hpp:707,262,274): one trial field and one domain on the same space.
template <detail::FixedString Name, Integer D>
struct TrialField {
  const FiniteElementSpace<D>* fes;
};
template <detail::FixedString Name, Integer D>
struct IntegrationDomain {
  const FiniteElementSpace<D>* fes;
};
template <detail::FixedString Name, Integer D>
TrialField<Name, D> MakeTrialField(const FiniteElementSpace<D>& fes) {
  return {&fes};
}
template <detail::FixedString Name, Integer D>
IntegrationDomain<Name, D> MakeIntegrationDomain(const FiniteElementSpace<D>& fes) {
  return {&fes};
}
template <Integer D>
struct WeakFormContext {
  FiniteElementSpace<D> fes;
  std::string trial, domain;
};
template <detail::FixedString T, detail::FixedString M, Integer D>
WeakFormContext<D> MakeWeakFormContext(const TrialField<T, D>& u, const IntegrationDomain<M, D>& dom) {
  if (u.fes->handle() != dom.fes->handle())
    throw Error("MakeWeakFormContext: the trial field and the domain must share one space");
  return {*u.fes, T.str(), M.str()};
}

// ------------------------------------------------------------------------- operator plans
// What a recognised form (or a legacy factory) asks of the kernels; pure host data.
struct OperatorPlan {
  bool mass = false, cell = false, interior = false, boundary = false;
  std::shared_ptr<const detail::ScalarField> sigma;  // null: constant sigma_scale
  Real sigma_scale = 1.0;
  std::shared_ptr<const detail::VectorField> beta;
  std::shared_ptr<const detail::ScalarField> outflow;  // boundary indicator (null: 1)
  std::shared_ptr<const detail::ScalarField> inflow;   // legacy bc(X) (null: 0 or no boundary)
  const Real* beta_factor = nullptr;  // per-element velocity factor (device, num_elements; null: 1)
  // interior-penalty diffusion (MakeDiffusionOperator): diffusivity constant on each element
  bool diffusion = false;
  bool speed_of_light = false;  // y = x (MakeSpeedOfLightOperator)
  std::shared_ptr<const detail::ScalarField> diffusivity;
  Real ip_sigma = -1.0, ip_kappa = 0.0;
  std::string describe() const {
    if (diffusion) return "interior-penalty diffusion, diffusivity=" + (diffusivity ? diffusivity->name : "?");
    if (speed_of_light) return "speed of light (copy)";
    std::ostringstream s;
    s << (mass ? "mass" : "") << (mass && cell ? "+" : "") << (cell ? "cell" : "") << (interior ? "+interior" : "")
      << (boundary ? "+boundary" : "");
    if (mass) s << " sigma=" << (sigma ? sigma->name : "const") << "*" << sigma_scale;
    if (beta) s << " beta=" << beta->name;
    return s.str();
  }
};

namespace detail {

struct Factors {
  Real scale = 1.0;
  std::vector<NodeP> f;
};

inline void flatten(const NodeP& n, Factors& out) {
  switch (n->k) {
    case NK::Mul:
      flatten(n->a, out);
      flatten(n->b, out);
      return;
    case NK::Neg:
      out.scale = -out.scale;
      flatten(n->a, out);
      return;
    case NK::Scalar:
      out.scale *= n->value;
      return;
    default:
      out.f.push_back(n);
  }
}

inline void split_sum(const NodeP& n, Real sign, std::vector<std::pair<Real, NodeP>>& out) {
  if (n->k == NK::Add) {
    split_sum(n->a, sign, out);
    split_sum(n->b, sign, out);
  } else if (n->k == NK::Neg && n->a->k == NK::Add) {
    split_sum(n->a, -sign, out);
  } else {
    out.emplace_back(sign, n);
  }
}

inline std::string node_str(const NodeP& n) {
  switch (n->k) {
    case NK::Trial: return n->name;
    case NK::Test: return "test(" + n->name + ")";
    case NK::Grad: return "grad(" + node_str(n->a) + ")";
    case NK::Dot: return "dot(" + node_str(n->a) + ", " + node_str(n->b) + ")";
    case NK::Mul: return node_str(n->a) + " * " + node_str(n->b);
    case NK::Neg: return "-(" + node_str(n->a) + ")";
    case NK::Scalar: return std::to_string(n->value);
    case NK::Coef:
    case NK::VecCoef: return n->name;
    case NK::Normal: return "Normal";
    case NK::Jump: return "jump(" + node_str(n->a) + ")";
    case NK::Average: return "average(" + node_str(n->a) + ")";
    case NK::Upwind: return "upwind(" + node_str(n->a) + ", " + node_str(n->b) + ")";
    case NK::Add: return "(" + node_str(n->a) + " + " + node_str(n->b) + ")";
  }
  return "?";
}

struct Matcher {
  std::vector<NodeP> f;
  // removes one factor satisfying pred and returns it (or null)
  template <typename P>
  NodeP take(P pred) {
    for (size_t i = 0; i < f.size(); ++i)
      if (pred(f[i])) {
        NodeP n = f[i];
        f.erase(f.begin() + (long)i);
        return n;
      }
    return nullptr;
  }
};

inline bool is(const NodeP& n, NK k) { return n && n->k == k; }

// dot(beta, X) or dot(X, beta) with X matching pred: returns beta's node
template <typename P>
NodeP dot_with_beta(const NodeP& n, P pred) {
  if (!is(n, NK::Dot)) return nullptr;
  if (is(n->a, NK::VecCoef) && pred(n->b)) return n->a;
  if (is(n->b, NK::VecCoef) && pred(n->a)) return n->b;
  return nullptr;
}

}  // namespace detail

// Recognises the hot-path weak forms (see the top of this file).
inline OperatorPlan PlanWeakForm(const WeakForm& wf, const std::string& trial, const std::string& domain) {
  using namespace detail;
  OperatorPlan plan;
  auto fail = [](const std::string& why, const NodeP& e) {
    throw Error("MakeGenericOperator: " + why + (e ? " in term: " + node_str(e) : std::string()));
  };
  auto same_beta = [&](const NodeP& bn, const NodeP& e) {
    if (!plan.beta) plan.beta = bn->vf;
    else if (plan.beta != bn->vf) fail("all advection terms must use the same velocity coefficient", e);
  };
  auto is_trial = [&](const NodeP& n) { return is(n, NK::Trial) && n->name == trial; };
  auto is_test = [&](const NodeP& n) { return is(n, NK::Test) && n->name == trial; };
  for (const Integral& in : wf.terms) {
    if (in.domain != domain) fail("integration domain '" + in.domain + "' is not the context's '" + domain + "'", in.expr);
    std::vector<std::pair<Real, NodeP>> parts;
    split_sum(in.expr, 1.0, parts);
    for (auto& [sign, e] : parts) {
      Factors fs;
      fs.scale = sign;
      flatten(e, fs);
      Matcher m{fs.f};
      if (in.kind == DomainKind::Cells) {
        NodeP bn;
        if (NodeP d = m.take([&](const NodeP& n) {
              return (bn = dot_with_beta(n, [&](const NodeP& x) { return is(x, NK::Grad) && is_test(x->a); })) != nullptr;
            })) {
          if (!m.take(is_trial) || !m.f.empty()) fail("cell advection must be -u * dot(beta, grad(v))", e);
          if (fs.scale != -1.0) fail("cell advection must be -u * dot(beta, grad(v)) (coefficient -1)", e);
          if (plan.cell) fail("more than one cell advection term", e);
          same_beta(bn, e);
          plan.cell = true;
          continue;
        }
        if (!m.take(is_trial) || !m.take(is_test)) fail("unsupported cell term", e);
        NodeP c = m.take([](const NodeP& n) { return is(n, NK::Coef); });
        if (!m.f.empty()) fail("unsupported cell term", e);
        if (plan.mass) fail("more than one mass term", e);
        plan.mass = true;
        plan.sigma = c ? c->sf : nullptr;
        plan.sigma_scale = fs.scale;
      } else if (in.kind == DomainKind::InteriorFacets) {
        NodeP up = m.take([](const NodeP& n) { return is(n, NK::Upwind); });
        NodeP jv = m.take([&](const NodeP& n) { return is(n, NK::Jump) && is_test(n->a); });
        if (!up || !jv || !m.f.empty() || fs.scale != 1.0 || !is(up->a, NK::VecCoef) || !is_trial(up->b))
          fail("interior facet terms must be upwind(beta, u) * jump(v)", e);
        if (plan.interior) fail("more than one interior facet term", e);
        same_beta(up->a, e);
        plan.interior = true;
      } else {
        NodeP bn;
        NodeP d = m.take([&](const NodeP& n) {
          return (bn = dot_with_beta(n, [](const NodeP& x) { return is(x, NK::Normal); })) != nullptr;
        });
        if (!d || !m.take(is_trial) || !m.take(is_test) || fs.scale != 1.0)
          fail("boundary facet terms must be [outflow *] dot(beta, Normal{}) * u * v", e);
        NodeP c = m.take([](const NodeP& n) { return is(n, NK::Coef); });
        if (!m.f.empty()) fail("boundary facet terms must be [outflow *] dot(beta, Normal{}) * u * v", e);
        if (plan.boundary) fail("more than one boundary facet term", e);
        same_beta(bn, e);
        plan.boundary = true;
        plan.outflow = c ? c->sf : nullptr;
      }
    }
  }
  const bool adv = plan.cell || plan.interior || plan.boundary;
  if (adv && !(plan.cell && plan.interior))
    throw Error("MakeGenericOperator: an advection form needs both the cell term and the interior upwind term");
  if (!plan.mass && !adv) throw Error("MakeGenericOperator: empty weak form");
  return plan;
}

// ------------------------------------------------------------------------- operators
class SolverHandle {
 public:
  explicit SolverHandle(dgop_solver* s) : s_(s) {}
  ~SolverHandle() { dgop_solver_destroy(s_); }
  SolverHandle(const SolverHandle&) = delete;
  SolverHandle& operator=(const SolverHandle&) = delete;
  dgop_solver* get() const { return s_; }

 private:
  dgop_solver* s_;
};

template <Integer D>
class Operator {
 public:
  Operator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, const OperatorPlan& plan)
      : fes_(fes), plan_(plan), q_(ir.q) {
    create();
  }

  // y = A x, y overwritten (massoperator.hpp:209, advectionoperator.hpp:1070)
  void operator()(const Vector& x, Vector& y) const { Apply(x, y); }
  void Apply(const Vector& x, Vector& y) const {
    check_sizes(x, y);
    detail::check(dgop_apply(op_.get(), x.ReadDeviceData(), y.WriteDeviceData(), nullptr), "apply");
  }
  // y = A^T x (no reference counterpart)
  void ApplyTranspose(const Vector& x, Vector& y) const {
    check_sizes(x, y);
    detail::check(dgop_apply_transpose(op_.get(), x.ReadDeviceData(), y.WriteDeviceData(), nullptr), "apply transpose");
  }
  Integer Size() const { return fes_.GetNumberOfFiniteElementDofs(); }
  dgop_operator* handle() const { return op_.get(); }
  const OperatorPlan& plan() const { return plan_; }
  std::string KernelName() const {
    static const char* const names[] = {"generic", "kron", "kronnd", "diffusion", "copy"};
    const int k = dgop_operator_kernel(op_.get());
    return (k >= 0 && k < 5) ? names[k] : "unknown";
  }

  // device-resident solvers, created once per (kind, restart, inner precision); kind 0 CG,
  // 1 GMRES, 2 refinement GMRES, 3 a second GMRES handle (the adjoint solve's)
  dgop_solver* solver(int kind, int restart, int inner) const {
    const auto key = std::make_tuple(kind, restart, inner);
    auto it = solvers_.find(key);
    if (it != solvers_.end()) return it->second->get();
    dgop_solver* s = nullptr;
    if (kind == 0) detail::check(dgop_cg_create(op_.get(), &s), "ConjugateGradient");
    else if (kind == 1 || kind == 3) detail::check(dgop_gmres_create(op_.get(), restart, &s), "GMRES");
    else detail::check(dgop_gmres_ir_create(op_.get(), restart, inner, &s), "refinement GMRES");
    auto h = std::make_shared<SolverHandle>(s);
    solvers_[key] = h;
    return s;
  }

 private:
  FiniteElementSpace<D> fes_;
  OperatorPlan plan_;
  int q_;
  std::shared_ptr<dgop_operator> op_;
  mutable std::map<std::tuple<int, int, int>, std::shared_ptr<SolverHandle>> solvers_;

  void check_sizes(const Vector& x, const Vector& y) const {
    if (x.Size() != Size() || y.Size() != Size()) throw Error("operator: vector size does not match the space");
  }

  std::shared_ptr<Real> mu_;  // per-element diffusivity on the device (diffusion operators)

  // The Kronecker-form diffusion kernel takes one diffusivity per element: evaluate the
  // reference's function of X at every Gauss point of every element and require it constant
  // on each element.
  void create_diffusion(const detail::Grid& g) {
    const CartesianMesh<D>& mesh = fes_.GetMesh();
    int64_t ne = 1;
    for (Integer k = 0; k < D; ++k) ne *= (int64_t)mesh.sizes[k];
    std::vector<Real> mu((size_t)ne);
    const int q = q_;
    int64_t qd = 1;
    for (Integer k = 0; k < D; ++k) qd *= q;
    for (int64_t e = 0; e < ne; ++e) {
      int64_t c[D];
      int64_t r = e;
      for (Integer k = 0; k < D; ++k) {
        c[k] = r % (int64_t)mesh.sizes[k];
        r /= (int64_t)mesh.sizes[k];
      }
      Real first = 0.0;
      for (int64_t p = 0; p < qd; ++p) {
        Real X[6];
        int64_t t = p;
        for (Integer k = 0; k < D; ++k) {
          X[k] = g.x[k][c[k] * (q + 2) + t % q];
          t /= q;
        }
        const Real v = plan_.diffusivity->eval((int)D, X);
        if (p == 0) first = v;
        else if (std::abs(v - first) > 1e-14 * std::max(std::abs(first), Real(1)))
          throw Error("MakeDiffusionOperator: the diffusivity '" + plan_.diffusivity->name +
                      "' must be constant on each element");
      }
      mu[(size_t)e] = first;
    }
    Real* d = nullptr;
    if (cudaMalloc(&d, sizeof(Real) * (size_t)ne) != cudaSuccess) throw Error("MakeDiffusionOperator: cudaMalloc");
    mu_ = std::shared_ptr<Real>(d, [](Real* ptr) { cudaFree(ptr); });
    if (cudaMemcpy(d, mu.data(), sizeof(Real) * (size_t)ne, cudaMemcpyHostToDevice) != cudaSuccess)
      throw Error("MakeDiffusionOperator: cudaMemcpy");
    dgop_operator* op = nullptr;
    detail::check(dgop_sipdg_create(fes_.handle(), q_, d, plan_.ip_sigma, plan_.ip_kappa, 1, &op),
                  "operator creation (" + plan_.describe() + ")");
    op_ = std::shared_ptr<dgop_operator>(op, [](dgop_operator* o) { dgop_operator_destroy(o); });
  }

  void create() {
    const CartesianMesh<D>& mesh = fes_.GetMesh();
    int64_t n[D];
    int per[D];
    for (Integer k = 0; k < D; ++k) {
      n[k] = (int64_t)mesh.sizes[k];
      per[k] = mesh.is_periodic_boundary[k];
    }
    if (plan_.speed_of_light) {
      dgop_operator* op = nullptr;
      detail::check(dgop_speed_of_light_create(fes_.handle(), q_, &op), "operator creation (speed of light)");
      op_ = std::shared_ptr<dgop_operator>(op, [](dgop_operator* o) { dgop_operator_destroy(o); });
      return;
    }
    detail::Grid g = detail::make_grid(fes_.handle(), (int)D, n, per, q_);
    if (plan_.diffusion) {
      create_diffusion(g);
      return;
    }
    detail::Separated sig;
    dgop_coef sigma{};
    if (plan_.mass) {
      if (plan_.sigma) {
        auto f = plan_.sigma;
        const Real s = plan_.sigma_scale;
        sig = detail::separate(g, [&](const Real* X) { return s * f->eval((int)D, X); }, "mass coefficient '" + f->name + "'");
      } else {
        sig.constant = plan_.sigma_scale;
      }
      sig.fill(sigma);
    }
    std::array<detail::Separated, D> bsep;
    std::array<dgop_coef, D> beta{};
    Real g_in = 0.0;
    if (plan_.cell) {
      auto bf = plan_.beta;
      for (Integer c = 0; c < D; ++c) {
        bsep[c] = detail::separate(
            g,
            [&](const Real* X) {
              Real v[6];
              bf->eval((int)D, X, v);
              return v[c];
            },
            "velocity '" + bf->name + "' component " + std::to_string(c));
        bsep[c].fill(beta[c]);
        beta[c].element_factor = plan_.beta_factor;
      }
      if (plan_.boundary) g_in = check_boundary(g);
    }
    dgop_operator* op = nullptr;
    const dgop_space* sp = fes_.handle();
    int rc;
    if (plan_.mass && !plan_.cell) rc = dgop_mass_create(sp, q_, &sigma, &op);
    else if (!plan_.mass) rc = dgop_advection_create(sp, q_, beta.data(), plan_.boundary ? DGOP_BC_INFLOW : DGOP_BC_NONE, g_in, &op);
    else if (!plan_.boundary) rc = dgop_mass_advection_create(sp, q_, &sigma, beta.data(), &op);
    else rc = dgop_system_create(sp, q_, &sigma, beta.data(), DGOP_BC_INFLOW, g_in, &op);
    detail::check(rc, "operator creation (" + plan_.describe() + ")");
    op_ = std::shared_ptr<dgop_operator>(op, [](dgop_operator* o) { dgop_operator_destroy(o); });
  }

  // The boundary term must be the upwind flux: on outflow points (beta.n > 0) the weak form's
  // indicator is 1, on inflow points it is 0 (weak forms) or the legacy bc(X) is one constant.
  Real check_boundary(const detail::Grid& g) const {
    bool have_in = false;
    Real g_in = 0.0;
    std::string err;
    detail::for_boundary_points(g, [&](const Real* X, int axis, int side) {
      if (!err.empty()) return;
      Real v[6];
      plan_.beta->eval((int)D, X, v);
      const Real bn = side == 0 ? -v[axis] : v[axis];
      if (plan_.inflow) {
        if (bn < 0.0) {
          const Real gv = plan_.inflow->eval((int)D, X);
          if (have_in && gv != g_in) err = "the inflow boundary value must be one constant";
          have_in = true;
          g_in = gv;
        }
        return;
      }
      const Real c = plan_.outflow ? plan_.outflow->eval((int)D, X) : 1.0;
      if (bn > 0.0 && c != 1.0) err = "the boundary indicator must be 1 on outflow points";
      if (bn < 0.0 && c != 0.0) err = "the boundary term must vanish on inflow points (upwind outflow term)";
    });
    if (!err.empty()) throw Error("operator creation: " + err);
    return g_in;
  }
};

// ---- legacy factories (massoperator.hpp:270, advectionoperator.hpp:1416,1481,
//      massadvectionoperator.hpp:447)
template <typename KernelPolicy, Integer D, typename Sigma>
Operator<D> MakeMassFiniteElementOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir,
                                          const Sigma& sigma) {
  OperatorPlan p;
  p.mass = true;
  p.sigma = detail::make_scalar(sigma, "sigma");
  return Operator<D>(fes, ir, p);
}

template <typename KernelPolicy, Integer D, typename Adv>
Operator<D> MakeAdvectionOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, const Adv& adv) {
  OperatorPlan p;
  p.cell = p.interior = true;
  p.beta = detail::make_vector(adv, "adv");
  return Operator<D>(fes, ir, p);
}

template <typename KernelPolicy, Integer D, typename Adv, typename BC>
Operator<D> MakeAdvectionOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, const Adv& adv,
                                  const BC& bc) {
  OperatorPlan p;
  p.cell = p.interior = p.boundary = true;
  p.beta = detail::make_vector(adv, "adv");
  p.inflow = detail::make_scalar(bc, "boundary value");
  return Operator<D>(fes, ir, p);
}

template <typename KernelPolicy, Integer D, typename Adv, typename Sigma>
Operator<D> MakeMassAdvectionOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, const Adv& adv,
                                      const Sigma& sigma) {
  OperatorPlan p;
  p.mass = p.cell = p.interior = true;
  p.sigma = detail::make_scalar(sigma, "sigma");
  p.beta = detail::make_vector(adv, "adv");
  return Operator<D>(fes, ir, p);
}

// MakeDiffusionOperator<KP>(fes, ir, velocity, sigma, kappa) (diffusionoperator.hpp:554): the
// legacy SIPDG operator with diffusivity velocity(X), penalty kappa / h, boundary faces included;
// here the diffusivity must be constant on each element.
template <typename KernelPolicy, Integer D, typename Velocity>
Operator<D> MakeDiffusionOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir,
                                  const Velocity& velocity, const Real sigma, const Real kappa) {
  OperatorPlan p;
  p.diffusion = true;
  p.diffusivity = detail::make_scalar(velocity, "velocity");
  p.ip_sigma = sigma;
  p.ip_kappa = kappa;
  return Operator<D>(fes, ir, p);
}

// MakeSpeedOfLightOperator<KP>(fes, ir) (speedoflightoperator.hpp:198): y = x element by
// element, the bandwidth reference of an apply.
template <typename KernelPolicy, Integer D>
Operator<D> MakeSpeedOfLightOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir) {
  OperatorPlan p;
  p.speed_of_light = true;
  return Operator<D>(fes, ir, p);
}

// (mass(sigma) + advection with inflow value bc) in one fused launch; no reference counterpart
// (the reference composes the two operators).
template <typename KernelPolicy, Integer D, typename Sigma, typename Adv, typename BC>
Operator<D> MakeMassPlusAdvectionOperator(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir,
                                          const Sigma& sigma, const Adv& adv, const BC& bc) {
  OperatorPlan p;
  p.mass = p.cell = p.interior = p.boundary = true;
  p.sigma = detail::make_scalar(sigma, "sigma");
  p.beta = detail::make_vector(adv, "adv");
  p.inflow = detail::make_scalar(bc, "boundary value");
  return Operator<D>(fes, ir, p);
}

// MakeGenericOperator<KP>(weak_form, context, integration_rule) (genericoperator.hpp:138)
template <typename KernelPolicy, Integer D>
Operator<D> MakeGenericOperator(const WeakForm& wf, const WeakFormContext<D>& ctx, const IntegrationRule<D>& ir) {
  return Operator<D>(ctx.fes, ir, PlanWeakForm(wf, ctx.trial, ctx.domain));
}

// ------------------------------------------------------------------------- Krylov drivers
// IterativeSolverResult (Solvers/iterativesolverresult.hpp:41)
struct IterativeSolverResult {
  bool success;
  Integer iterations;
  Real relative_error;
};

namespace detail {
inline IterativeSolverResult solve(dgop_solver* s, const Vector& rhs, Vector& x, Integer max_iters, Real tol) {
  if (rhs.Size() != x.Size()) throw Error("solver: vector sizes do not match");
  dgop_solve_result r{};
  check(dgop_solver_solve(s, rhs.ReadDeviceData(), x.ReadWriteDeviceData(), (int)max_iters, tol, &r, nullptr), "solve");
  return {r.success != 0, (Integer)r.iterations, r.relative_error};
}
}  // namespace detail

// ConjugateGradient scratch overload (conjugategradient.hpp:125-209), device resident: the dot
// functor and the scratch vectors are accepted for source compatibility; the solver's own
// deterministic device reductions and workspace are used.
template <Integer D, typename DotType>
IterativeSolverResult ConjugateGradient(const Operator<D>& A, const Vector& rhs, const DotType&, Integer max_iters,
                                        Real tol, Vector& x, Vector&, Vector&, Vector&, Vector&) {
  return detail::solve(A.solver(0, 0, 0), rhs, x, max_iters, tol);
}

// ConjugateGradient(kernel_conf, A, rhs, max_iters, tol, x) (conjugategradient.hpp:217)
template <typename KernelContext, Integer D>
IterativeSolverResult ConjugateGradient(KernelContext&, const Operator<D>& A, const Vector& rhs,
                                        const Integer& max_iters, const Real& tol, Vector& x) {
  return detail::solve(A.solver(0, 0, 0), rhs, x, max_iters, tol);
}

// GMRES_no_alloc (Solvers/gmres.hpp:74-289), device resident (workspace arguments as above).
template <Integer D, typename DotType, typename VectorArray, typename Array>
IterativeSolverResult GMRES_no_alloc(const Operator<D>& A, const Vector& rhs, const DotType&, const Integer max_iters,
                                     const Integer restart, const Real tol, Vector& x, VectorArray&, Vector&, Array&,
                                     Array&, Array&, Array&, Array&) {
  return detail::solve(A.solver(1, (int)restart, 0), rhs, x, max_iters, tol);
}

// GMRES(restart) with FP32 (or FP64) inner cycles and FP64 iterative refinement; same stopping
// test and result as GMRES_no_alloc.  No reference counterpart.
template <Integer D>
IterativeSolverResult RefinedGMRES(const Operator<D>& A, const Vector& rhs, Integer max_iters, Integer restart,
                                   Real tol, Vector& x, bool fp32_inner = true) {
  return detail::solve(A.solver(2, (int)restart, fp32_inner ? DGOP_FP32 : DGOP_FP64), rhs, x, max_iters, tol);
}

// ------------------------------------------------------------------------- adjoint gradients
// Forward/backward pair for u = S(theta)^{-1} b with S(theta) = M_sigma + A(theta_e beta(X)) and
// inflow value bc (one constant): theta holds one velocity factor per element.  Backward gives,
// for an upstream gradient dJ/du, dJ/db = S^{-T} dJ/du and
//   dJ/dtheta_e = -s_e (dJ/db)_e . (A(s beta) u)_e,   s_e = sign(theta_e),
// because the rows of element e depend on theta_e alone (own cell term and own face fluxes).
// Forward and adjoint solves run GMRES(restart) on the device; no Krylov iterate is stored.  No
// reference counterpart.
template <Integer D>
class AdvectionSolveFunction {
 public:
  template <typename Sigma, typename Adv, typename BC>
  AdvectionSolveFunction(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, const Sigma& sigma,
                         const Adv& adv, const BC& bc, Integer restart = 30, Real tol = 1e-12,
                         Integer max_iters = 20000)
      : fes_(fes), ir_(ir), restart_(restart), tol_(tol), max_iters_(max_iters) {
    plan_.mass = plan_.cell = plan_.interior = plan_.boundary = true;
    plan_.sigma = detail::make_scalar(sigma, "sigma");
    plan_.beta = detail::make_vector(adv, "adv");
    plan_.inflow = detail::make_scalar(bc, "boundary value");
  }

  IterativeSolverResult Forward(const Vector& theta, const Vector& b, Vector& u) {
    theta_ = theta;
    u_ = Vector(b.Size());
    u_ = 0.0;
    op_ = std::make_unique<Operator<D>>(fes_, ir_, with_factor(plan_, theta_.ReadDeviceData()));
    const IterativeSolverResult r =
        detail::solve(op_->solver(1, (int)restart_, 0), b, u_, max_iters_, tol_);
    u = u_;
    return r;
  }

  IterativeSolverResult Backward(const Vector& grad_u, Vector& grad_theta, Vector& grad_b) {
    if (!op_) throw Error("AdvectionSolveFunction: Backward before Forward");
    dgop_solver* adj = op_->solver(3, (int)restart_, 0);
    grad_b = Vector(grad_u.Size());
    grad_b = 0.0;
    detail::check(dgop_solver_set_transpose(adj, 1), "adjoint solve");
    const IterativeSolverResult r = detail::solve(adj, grad_u, grad_b, max_iters_, tol_);
    // s = sign(theta) and the advection part with element factors s
    const Integer ne = fes_.GetNumberOfFiniteElements();
    Vector s(ne);
    {
      const Real* t = theta_.ReadHostData();
      Real* sp = s.WriteHostData();
      for (Integer e = 0; e < ne; ++e) sp[e] = t[e] < 0.0 ? -1.0 : 1.0;
    }
    OperatorPlan adv = plan_;
    adv.mass = false;
    Operator<D> A(fes_, ir_, with_factor(adv, s.ReadDeviceData()));
    Vector w(u_.Size());
    A(u_, w);
    grad_theta = Vector(ne);
    detail::check(dgop_element_dot(A.handle(), grad_b.ReadDeviceData(), w.ReadDeviceData(), s.ReadDeviceData(),
                                   grad_theta.WriteDeviceData(), nullptr),
                  "element products");
    grad_theta *= -1.0;
    return r;
  }

 private:
  static OperatorPlan with_factor(OperatorPlan p, const Real* factor) {
    p.beta_factor = factor;
    return p;
  }
  FiniteElementSpace<D> fes_;
  IntegrationRule<D> ir_;
  Integer restart_;
  Real tol_;
  Integer max_iters_;
  OperatorPlan plan_;
  Vector theta_, u_;
  std::unique_ptr<Operator<D>> op_;
};

// Solve-based loss gradients for the interior-penalty DG diffusion operator with one
// diffusivity per element, A(mu) u = f: the reference's SIPDG weak form with a per-element
// coefficient field (tests/integration/gendil/test-sipdg-coefficient-field-inputs.cpp:547-569),
// symmetric (sigma = -1), penalty kappa / h, Dirichlet-0 boundary terms when `boundary`.
//   Forward(mu, f, u):  u = A(mu)^{-1} f by CG on the device.
//   Backward(dJ/du, dJ/dmu, dJ/df):  lambda = A^{-1} dJ/du (A^T = A), then
//     dJ/dmu_e = -lambda^T (dA/dmu_e) u   (dgop_sipdg_gradient: one kernel over all elements),
//     dJ/df = lambda.
// A is linear in mu and each element's diffusivity enters only its own rows and its faces' rows,
// which the gradient kernel sums.  Forward keeps u and the operator; no Krylov iterate is stored.
// No reference counterpart.
template <Integer D>
class DiffusionSolveFunction {
 public:
  DiffusionSolveFunction(const FiniteElementSpace<D>& fes, const IntegrationRule<D>& ir, Real kappa,
                         bool boundary = true, Real tol = 1e-12, Integer max_iters = 100000)
      : fes_(fes), q_(ir.q), kappa_(kappa), boundary_(boundary), tol_(tol), max_iters_(max_iters) {}

  IterativeSolverResult Forward(const Vector& mu, const Vector& f, Vector& u) {
    if (mu.Size() != fes_.GetNumberOfFiniteElements()) throw Error("DiffusionSolveFunction: one mu per element");
    mu_ = mu;
    release();
    detail::check(dgop_sipdg_create(fes_.handle(), q_, mu_.ReadDeviceData(), -1.0, kappa_, boundary_ ? 1 : 0, &op_),
                  "DiffusionSolveFunction operator");
    detail::check(dgop_cg_create(op_, &cg_), "DiffusionSolveFunction CG");
    u_ = Vector(f.Size());
    u_ = 0.0;
    const IterativeSolverResult r = detail::solve(cg_, f, u_, max_iters_, tol_);
    u = u_;
    return r;
  }

  IterativeSolverResult Backward(const Vector& grad_u, Vector& grad_mu, Vector& grad_f) {
    if (!op_) throw Error("DiffusionSolveFunction: Backward before Forward");
    grad_f = Vector(grad_u.Size());
    grad_f = 0.0;
    const IterativeSolverResult r = detail::solve(cg_, grad_u, grad_f, max_iters_, tol_);
    grad_mu = Vector(fes_.GetNumberOfFiniteElements());
    detail::check(dgop_sipdg_gradient(op_, u_.ReadDeviceData(), grad_f.ReadDeviceData(), nullptr,
                                      grad_mu.WriteDeviceData(), nullptr),
                  "coefficient gradient");
    grad_mu *= -1.0;
    return r;
  }

  ~DiffusionSolveFunction() { release(); }
  DiffusionSolveFunction(const DiffusionSolveFunction&) = delete;
  DiffusionSolveFunction& operator=(const DiffusionSolveFunction&) = delete;

 private:
  void release() {
    if (cg_) dgop_solver_destroy(cg_);
    if (op_) dgop_operator_destroy(op_);
    cg_ = nullptr;
    op_ = nullptr;
  }
  FiniteElementSpace<D> fes_;
  int q_;
  Real kappa_;
  bool boundary_;
  Real tol_;
  Integer max_iters_;
  Vector mu_, u_;
  dgop_operator* op_ = nullptr;
  dgop_solver* cg_ = nullptr;
};

}  // namespace gendil_b200
