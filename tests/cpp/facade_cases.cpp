// Cases for the C++20 facade (include/gendil_b200/gendil.hpp), written the way GenDiL's own
// integration tests use the library (tests/integration/gendil/test-advection-3d-generic.cpp,
// test-mass-3d-generic.cpp): meshes, spaces, rules, legacy factories, weak forms, solvers.
//
//   facade_cases plan          host only: weak-form recognition and coefficient separation
//   facade_cases run <file>    GPU: applies and solves; every result vector is appended to <file>
//                              as [u32 name length][name][u64 n][n doubles], and one line
//                              "solve <name> <success> <iterations> <relative error>" per solve
//                              goes to stdout
// The test driver compares the vectors with the oracle.
#include <gendil_b200/gendil.hpp>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>

using namespace gendil_b200;

namespace {

FILE* g_out = nullptr;

void record(const std::string& name, const Vector& v) {
  const uint32_t len = (uint32_t)name.size();
  const uint64_t n = v.Size();
  std::fwrite(&len, sizeof(len), 1, g_out);
  std::fwrite(name.data(), 1, len, g_out);
  std::fwrite(&n, sizeof(n), 1, g_out);
  std::fwrite(v.ReadHostData(), sizeof(Real), n, g_out);
}

void report(const std::string& name, const IterativeSolverResult& r) {
  std::printf("solve %s %d %zu %.17g\n", name.c_str(), r.success ? 1 : 0, (size_t)r.iterations, r.relative_error);
}

// coefficient functions of the oracle's presets
auto sigma_poly = [](const std::array<Real, 3>& X) { return 1.0 + X[0] * X[1] + X[2] * X[2]; };
auto sigma_sep = [](const std::array<Real, 3>& X) { return (1.0 + 0.5 * X[0]) * (1.0 + X[1] * X[1]) * (2.0 - X[2]); };
auto beta_sincos = [](const std::array<Real, 3>& X) -> std::array<Real, 3> {
  return {1.0 + 0.5 * std::sin(2.0 * M_PI * X[1]), 0.5 + 0.25 * std::cos(2.0 * M_PI * X[2]), 0.25};
};
auto adv_sincos = [](const std::array<Real, 3>& X, Real (&v)[3]) {
  const auto b = beta_sincos(X);
  for (int d = 0; d < 3; ++d) v[d] = b[d];
};
auto adv_bubble = [](const std::array<Real, 3>& X, Real (&v)[3]) {
  for (int d = 0; d < 3; ++d) v[d] = -X[d] * (1.0 - X[d]);
};
auto zero3 = [](const std::array<Real, 3>&) { return 0.0; };
// the sin/cos velocity leaves through x = 1, y = 1 and z = 1
auto outflow_sincos = [](const std::array<Real, 3>& X) {
  return (X[0] == 1.0 || X[1] == 1.0 || X[2] == 1.0) ? 1.0 : 0.0;
};

int plan_mode() {
  TrialSpace<"u"> u;
  TestSpace<"u"> v;
  Cells<"mesh"> cells;
  InteriorFacets<"mesh"> interior_facets;
  BoundaryFacets<"mesh"> boundary_facets;
  auto beta = MakeVectorCoefficient<"beta", PhysicalCoordinate>(beta_sincos);
  auto sigma = MakeCoefficient<"sigma", PhysicalCoordinate>(sigma_poly);
  auto outflow = MakeCoefficient<"outflow", PhysicalCoordinate>(outflow_sincos);
  struct Case {
    const char* name;
    WeakForm wf;
  };
  const Real dt = 1e-3;
  Case cases[] = {
      {"mass", integrate(cells, u * v)},
      {"mass_coef", integrate(cells, sigma * u * v)},
      {"mass_scaled", integrate(cells, (1.0 / dt) * u * v)},
      {"advection", integrate(cells, -u * dot(beta, grad(v))) + integrate(interior_facets, upwind(beta, u) * jump(v))},
      {"advection_outflow", integrate(cells, -u * dot(beta, grad(v))) +
                                integrate(interior_facets, upwind(beta, u) * jump(v)) +
                                integrate(boundary_facets, outflow * dot(beta, Normal{}) * u * v)},
      {"system", integrate(cells, (1.0 / dt) * u * v - u * dot(beta, grad(v))) +
                     integrate(interior_facets, upwind(beta, u) * jump(v)) +
                     integrate(boundary_facets, outflow * dot(beta, Normal{}) * u * v)},
      {"reject_cell_only", integrate(cells, -u * dot(beta, grad(v)))},
      {"reject_wrong_sign", integrate(cells, u * dot(beta, grad(v))) + integrate(interior_facets, upwind(beta, u) * jump(v))},
      {"reject_grad_grad", integrate(cells, dot(grad(u), grad(v)))},
      {"reject_average", integrate(cells, -u * dot(beta, grad(v))) + integrate(interior_facets, average(u) * jump(v))},
      {"reject_two_mass", integrate(cells, u * v) + integrate(cells, sigma * u * v)},
  };
  for (auto& c : cases) {
    try {
      OperatorPlan p = PlanWeakForm(c.wf, "u", "mesh");
      std::printf("plan %s %s\n", c.name, p.describe().c_str());
    } catch (const Error& e) {
      std::printf("rejected %s: %s\n", c.name, e.what());
    }
  }
  // coefficient separation on the 8^3, q = 4 sample grid
  CartesianMesh<3> mesh({8, 8, 8}, {0.125, 0.125, 0.125}, {0.0, 0.0, 0.0});
  auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3, 3>{}));
  int64_t n[3] = {8, 8, 8};
  int per[3] = {0, 0, 0};
  detail::Grid g = detail::make_grid(fes.handle(), 3, n, per, 4);
  auto as_fn = [](auto f) {
    return std::function<Real(const Real*)>([f](const Real* X) { return f(std::array<Real, 3>{X[0], X[1], X[2]}); });
  };
  struct Sep {
    const char* name;
    std::function<Real(const Real*)> f;
  };
  Sep seps[] = {
      {"const", as_fn([](const std::array<Real, 3>&) { return 2.5; })},
      {"one_axis", as_fn([](const std::array<Real, 3>& X) { return 0.5 + 0.25 * std::cos(2.0 * M_PI * X[2]); })},
      {"poly", as_fn(sigma_poly)},
      {"sep", as_fn(sigma_sep)},
      {"additive", as_fn([](const std::array<Real, 3>& X) { return std::exp(X[0]) + X[1] * X[1] - std::sin(X[2]); })},
      {"reject_nonsep", as_fn([](const std::array<Real, 3>& X) { return std::exp(X[0] * X[1] * X[2]) + X[0] * X[1]; })},
  };
  for (auto& s : seps) {
    try {
      detail::Separated r = detail::separate(g, s.f, s.name);
      std::printf("separated %s terms=%zu\n", s.name, r.terms.size());
    } catch (const Error& e) {
      std::printf("rejected %s: %s\n", s.name, e.what());
    }
  }
  return 0;
}

int run_mode(const char* path) {
  g_out = std::fopen(path, "wb");
  if (!g_out) return 2;
  TrialSpace<"u"> u;
  TestSpace<"u"> v;
  Cells<"mesh"> cells;
  InteriorFacets<"mesh"> interior_facets;
  BoundaryFacets<"mesh"> boundary_facets;
  using KernelPolicy = DeviceKernelConfiguration;

  {  // A: mass, sigma = 1 + x y + z^2, 8^3, p = 3, q = 4: legacy and weak form
    CartesianMesh<3> mesh({8, 8, 8}, {0.125, 0.125, 0.125}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3, 3>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    Vector x(fes), y(fes), z(fes);
    FillRandom(x, 0);
    auto mass = MakeMassFiniteElementOperator<KernelPolicy>(fes, ir, sigma_poly);
    mass(x, y);
    record("A_legacy", y);
    auto sigma = MakeCoefficient<"sigma", PhysicalCoordinate>(sigma_poly);
    auto ctx = MakeWeakFormContext(MakeTrialField<"u">(fes), MakeIntegrationDomain<"mesh">(fes));
    auto op = MakeGenericOperator<KernelPolicy>(integrate(cells, sigma * u * v), ctx, ir);
    op(x, z);
    record("A_generic", z);
  }
  {  // B: mass, sigma = (1 + x/2)(1 + y^2)(2 - z), 6^3, p = 2, q = 3
    CartesianMesh<3> mesh({6, 6, 6}, {1.0 / 6, 1.0 / 6, 1.0 / 6}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<2, 2, 2>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<3, 3, 3>{});
    Vector x(fes), y(fes);
    FillRandom(x, 0);
    MakeMassFiniteElementOperator<KernelPolicy>(fes, ir, sigma_sep)(x, y);
    record("B_legacy", y);
  }
  {  // C: advection with the sin/cos velocity, 8^3, p = 3, q = 4
    CartesianMesh<3> mesh({8, 8, 8}, {0.125, 0.125, 0.125}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3, 3>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    Vector x(fes), y(fes);
    FillRandom(x, 1);
    MakeAdvectionOperator<KernelPolicy>(fes, ir, adv_sincos, zero3)(x, y);
    record("C_legacy_bc", y);
    MakeAdvectionOperator<KernelPolicy>(fes, ir, adv_sincos)(x, y);
    record("C_legacy_nobc", y);
    auto beta = MakeVectorCoefficient<"beta", PhysicalCoordinate>(beta_sincos);
    auto outflow = MakeCoefficient<"outflow", PhysicalCoordinate>(outflow_sincos);
    auto ctx = MakeWeakFormContext(MakeTrialField<"u">(fes), MakeIntegrationDomain<"mesh">(fes));
    auto form = integrate(cells, -u * dot(beta, grad(v))) + integrate(interior_facets, upwind(beta, u) * jump(v));
    MakeGenericOperator<KernelPolicy>(form, ctx, ir)(x, y);
    record("C_generic_nobc", y);
    auto form_bc = form + integrate(boundary_facets, outflow * dot(beta, Normal{}) * u * v);
    MakeGenericOperator<KernelPolicy>(form_bc, ctx, ir)(x, y);
    record("C_generic_bc", y);
  }
  {  // D: mass + advection (interior faces only), bubble velocity, sigma = 10, 6^3, p = 2, q = 3
    CartesianMesh<3> mesh({6, 6, 6}, {1.0 / 6, 1.0 / 6, 1.0 / 6}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<2, 2, 2>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<3, 3, 3>{});
    Vector x(fes), y(fes);
    FillRandom(x, 1);
    auto ten = [](const std::array<Real, 3>&) { return 10.0; };
    MakeMassAdvectionOperator<KernelPolicy>(fes, ir, adv_bubble, ten)(x, y);
    record("D_legacy", y);
  }
  {  // E: 2D advection, constant velocity (0.7, -0.4), inflow value 0.75, 7 x 9, p = 4, q = 5
    CartesianMesh<2> mesh({7, 9}, {1.0 / 7, 1.0 / 9}, {0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<4, 4>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<5, 5>{});
    Vector x(fes), y(fes);
    FillRandom(x, 1);
    auto adv = [](const std::array<Real, 2>&, Real (&w)[2]) {
      w[0] = 0.7;
      w[1] = -0.4;
    };
    auto g = [](const std::array<Real, 2>&) { return 0.75; };
    MakeAdvectionOperator<KernelPolicy>(fes, ir, adv, g)(x, y);
    record("E_legacy_bc", y);
  }
  {  // F: CG on the 16^3 p = 3 mass matrix, b = M u (u from seed 0), 20 iterations, tol 1e-6
    CartesianMesh<3> mesh({16, 16, 16}, {1.0 / 16, 1.0 / 16, 1.0 / 16}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3, 3>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    auto one = [](const std::array<Real, 3>&) { return 1.0; };
    auto mass = MakeMassFiniteElementOperator<KernelPolicy>(fes, ir, one);
    Vector uu(fes), b(fes), x(fes), tmp(fes), zz(fes), r(fes), p(fes);
    FillRandom(uu, 0);
    mass(uu, b);
    x = 0.0;
    auto dot = [](const Vector& a, const Vector& c) { return Dot(a, c); };
    report("F_cg", ConjugateGradient(mass, b, dot, 20, 1e-6, x, tmp, zz, r, p));
    record("F_cg_x", x);
  }
  {  // G: GMRES(30) on (M/dt + A) x = b, 4^3, p = 3, q = 4, sin/cos velocity, outflow boundary term
    const Real dt = 1e-3;
    CartesianMesh<3> mesh({4, 4, 4}, {0.25, 0.25, 0.25}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3, 3>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    auto beta = MakeVectorCoefficient<"beta", PhysicalCoordinate>(beta_sincos);
    auto outflow = MakeCoefficient<"outflow", PhysicalCoordinate>(outflow_sincos);
    auto form = integrate(cells, (1.0 / dt) * u * v - u * dot(beta, grad(v))) +
                integrate(interior_facets, upwind(beta, u) * jump(v)) +
                integrate(boundary_facets, outflow * dot(beta, Normal{}) * u * v);
    auto ctx = MakeWeakFormContext(MakeTrialField<"u">(fes), MakeIntegrationDomain<"mesh">(fes));
    auto A = MakeGenericOperator<KernelPolicy>(form, ctx, ir);
    Vector b(fes), x(fes), w(fes);
    FillRandom(b, 2);
    x = 0.0;
    std::vector<Vector> V(31, Vector(fes));
    std::vector<Real> H(31 * 30), cs(30), sn(30), e1(31), yv(30);
    auto dot = [](const Vector& a, const Vector& c) { return Dot(a, c); };
    report("G_gmres", GMRES_no_alloc(A, b, dot, 5000, 30, 1e-10, x, V, w, H, cs, sn, e1, yv));
    record("G_gmres_x", x);
    x = 0.0;
    report("G_refined", RefinedGMRES(A, b, 5000, 30, 1e-10, x));
    record("G_refined_x", x);
  }
  {  // H: adjoint gradient of J = |u - u*|^2 / 2 w.r.t. per-element velocity factors, with
     // central differences through the forward solve
    CartesianMesh<3> mesh({3, 3, 2}, {1.0 / 3, 1.0 / 3, 0.5}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<2, 2, 2>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<3, 3, 3>{});
    auto sigma = [](const std::array<Real, 3>&) { return 20.0; };
    auto g_in = [](const std::array<Real, 3>&) { return 0.3; };
    AdvectionSolveFunction<3> fn(fes, ir, sigma, adv_sincos, g_in, 30, 1e-14);
    const Integer ne = fes.GetNumberOfFiniteElements();
    Vector theta(ne), b(fes), target(fes), u(fes);
    FillRandom(theta, 11, 0.5, 1.5);
    FillRandom(b, 5);
    FillRandom(target, 6);
    auto loss = [&](const Vector& th) {
      Vector uu(fes);
      fn.Forward(th, b, uu);
      Real J = 0.0;
      for (Integer i = 0; i < uu.Size(); ++i) J += 0.5 * (uu[i] - target[i]) * (uu[i] - target[i]);
      return J;
    };
    report("H_forward", fn.Forward(theta, b, u));
    Vector grad_u(fes), grad_theta, grad_b;
    for (Integer i = 0; i < u.Size(); ++i) grad_u[i] = u[i] - target[i];
    report("H_adjoint", fn.Backward(grad_u, grad_theta, grad_b));
    Real gmax = 0.0, worst = 0.0;
    for (Integer e = 0; e < ne; ++e) gmax = std::max(gmax, std::fabs(grad_theta[e]));
    const Real eps = 1e-6;
    for (Integer e : {Integer(0), Integer(5), Integer(9), ne - 1}) {
      Vector tp = theta, tm = theta;
      tp[e] += eps;
      tm[e] -= eps;
      const Real fd = (loss(tp) - loss(tm)) / (2 * eps);
      worst = std::max(worst, std::fabs(fd - grad_theta[e]));
    }
    std::printf("check H_fd %.6g\n", worst / gmax);
    record("H_grad_theta", grad_theta);
  }
  {  // K: adjoint gradient of J = |u - u*|^2 / 2 w.r.t. per-element diffusivities of the SIPDG
     // operator (DiffusionSolveFunction), with central differences through the forward solve;
     // J(mu+) - J(mu-) = (u+ - u-) . (u+ + u- - 2 u*) / 2 keeps the difference free of cancellation
    CartesianMesh<3> mesh({3, 3, 2}, {1.0 / 3, 1.0 / 3, 0.5}, {0.0, 0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<2, 2, 2>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    DiffusionSolveFunction<3> fn(fes, ir, 90.0, true, 1e-13);
    const Integer ne = fes.GetNumberOfFiniteElements();
    Vector mu(ne), f(fes), target(fes), u(fes);
    FillRandom(mu, 12, 0.5, 2.0);
    FillRandom(f, 5);
    FillRandom(target, 6);
    report("K_forward", fn.Forward(mu, f, u));
    Vector grad_u(fes), grad_mu, grad_f;
    for (Integer i = 0; i < u.Size(); ++i) grad_u[i] = u[i] - target[i];
    report("K_adjoint", fn.Backward(grad_u, grad_mu, grad_f));
    const Real eps = 1e-6;
    Real worst = 0.0;
    for (Integer e = 0; e < ne; ++e) {
      Vector mp = mu, mm = mu, up(fes), um(fes);
      mp[e] += eps;
      mm[e] -= eps;
      fn.Forward(mp, f, up);
      fn.Forward(mm, f, um);
      Real dj = 0.0;
      for (Integer i = 0; i < up.Size(); ++i) dj += 0.5 * (up[i] - um[i]) * (up[i] + um[i] - 2.0 * target[i]);
      worst = std::max(worst, std::fabs(dj / (2 * eps) - grad_mu[e]) / std::fabs(grad_mu[e]));
    }
    std::printf("check K_fd_rel %.6g\n", worst);
    record("K_grad_mu", grad_mu);
  }
  {  // I: legacy interior-penalty diffusion, MakeDiffusionOperator(fes, ir, velocity, sigma, kappa):
     // periodic 3^3, p = 2, q = 4, diffusivity 2.5, sigma = -1, kappa = 90 (golden case d4)
    CartesianMesh<3> mesh({3, 3, 3}, {1.0 / 3, 1.0 / 3, 1.0 / 3}, {0.0, 0.0, 0.0}, true);
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<2, 2, 2>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4, 4>{});
    auto velocity = [](const std::array<Real, 3>&) { return 2.5; };
    Vector x(fes), y(fes);
    FillRandom(x, 5);
    auto A = MakeDiffusionOperator<KernelPolicy>(fes, ir, velocity, -1.0, 90.0);
    A(x, y);
    record("I_diffusion", y);
    std::printf("check I_kernel_is_diffusion %d\n", A.KernelName() == "diffusion" ? 1 : 0);
    auto varying = [](const std::array<Real, 3>& X) { return 1.0 + X[0]; };
    try {
      MakeDiffusionOperator<KernelPolicy>(fes, ir, varying, -1.0, 90.0);
      std::printf("check I_rejects_varying 0\n");
    } catch (const Error&) {
      std::printf("check I_rejects_varying 1\n");
    }
  }
  {  // J: speed-of-light operator (y = x), 2D 5 x 4, p = 3
    CartesianMesh<2> mesh({5, 4}, {0.2, 0.25}, {0.0, 0.0});
    auto fes = MakeFiniteElementSpace(mesh, MakeLobattoFiniteElement(FiniteElementOrders<3, 3>{}));
    auto ir = MakeIntegrationRule(IntegrationRuleNumPoints<4, 4>{});
    Vector x(fes), y(fes);
    FillRandom(x, 3);
    auto sol = MakeSpeedOfLightOperator<KernelPolicy>(fes, ir);
    sol(x, y);
    bool same = true;
    for (Integer i = 0; i < x.Size(); ++i) same = same && (x[i] == y[i]);
    std::printf("check J_copy_exact %d\n", same ? 1 : 0);
  }
  std::fclose(g_out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    if (argc >= 2 && std::strcmp(argv[1], "plan") == 0) return plan_mode();
    if (argc >= 3 && std::strcmp(argv[1], "run") == 0) return run_mode(argv[2]);
  } catch (const Error& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "usage: facade_cases plan | run <file>\n");
  return 2;
}
