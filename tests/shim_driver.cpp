// shim_driver.cpp -- a C++ caller of include/dndsg_shim.hpp, built and run by tests/test_shim.py.
//
// It drives the GPU path through the reference-named classes in the order of the reference's
// explicit solver (DNDS_FV_EulerSolver.hpp:713-837 frhs, DNDS_ODE.hpp:131-177 SSP-RK3):
//   VRFiniteVolume2DGPU::ReconstructionJacobiStep x3 -> EulerEvaluatorGPU::EvaluateDt ->
//   EulerEvaluatorGPU::EvaluateRHS, then from the initial state with a zero reconstruction
//   two ExplicitSSPRK3GPU::Step calls.
//
// usage: shim_driver <input> <output>
// input (little-endian binary): int64 n_nodes, n_cells, n_faces; double node_xy[n_nodes][2];
//   int32 cell_nodes[n_cells][4], face_nodes[n_faces][2], face_cells[n_faces][2], face_bc[n_faces];
//   double face_shift[n_faces][2]; dndsg_settings (raw bytes); double u0[n_cells][4];
//   double cfl, t_rhs
// output: double dtmin, dt[n_cells], rhs[n_cells][4], u_rk2[n_cells][4], t_rk2
#include <cstdio>
#include <vector>

#include "dndsg_shim.hpp"

namespace {
template <class T>
bool read_into(std::FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return std::fread(v.data(), sizeof(T), n, f) == n;
}
template <class T>
void write_from(std::FILE* f, const T* p, size_t n) {
  std::fwrite(p, sizeof(T), n, f);
}
}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  std::FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int64_t n[3];
  if (std::fread(n, sizeof(int64_t), 3, in) != 3) return 2;
  const size_t nn = (size_t)n[0], nc = (size_t)n[1], nf = (size_t)n[2];
  std::vector<double> xy, shift, u0;
  std::vector<int32_t> cn, fn, fc, fb;
  dndsg_settings st{};
  double cfl = 0, tRhs = 0;
  bool ok = read_into(in, xy, 2 * nn) && read_into(in, cn, 4 * nc) && read_into(in, fn, 2 * nf) &&
            read_into(in, fc, 2 * nf) && read_into(in, fb, nf) && read_into(in, shift, 2 * nf) &&
            std::fread(&st, sizeof(st), 1, in) == 1 && read_into(in, u0, 4 * nc) &&
            std::fread(&cfl, sizeof(double), 1, in) == 1 && std::fread(&tRhs, sizeof(double), 1, in) == 1;
  std::fclose(in);
  if (!ok) {
    std::fprintf(stderr, "short input\n");
    return 2;
  }
  dndsg_mesh_desc md{(int64_t)nn, (int64_t)nc, (int64_t)nf, xy.data(), cn.data(), fn.data(), fc.data(), fb.data(),
                     shift.data()};
  try {
    dndsg::Context ctx(md, st, 0);
    dndsg::VRFiniteVolume2DGPU vfv(ctx);
    dndsg::EulerEvaluatorGPU eval(ctx);
    dndsg::ExplicitSSPRK3GPU ode(ctx);

    ctx.PushState(u0);
    vfv.ReconstructionJacobiStep(3);
    std::vector<double> dt, rhs;
    double dtMin = 0;
    eval.EvaluateDt(dt, cfl, dtMin, 1e100, false);
    eval.EvaluateRHS(rhs, tRhs);

    std::vector<double> zero(20 * nc, 0.0), u2;
    ctx.PushState(u0, &zero);
    ctx.check(dndsg_set_time(ctx.get(), 0.0, nullptr));
    ode.Step(cfl);
    ode.Step(cfl);
    ctx.PullState(u2);
    double t2 = 0;
    ctx.check(dndsg_get_time(ctx.get(), &t2, nullptr));

    std::FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    write_from(out, &dtMin, 1);
    write_from(out, dt.data(), nc);
    write_from(out, rhs.data(), 4 * nc);
    write_from(out, u2.data(), 4 * nc);
    write_from(out, &t2, 1);
    std::fclose(out);
  } catch (const dndsg::Error& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
