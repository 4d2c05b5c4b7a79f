// Host check of the face basis record (dndsg_bodies.cuh): the device headers compile as plain C++,
// so the setup (setup_cell, setup_face) and the record's expansion (FaceBasisSide::at) run here on
// the CPU.  For every face, side and Gauss point the record's basis values are compared with the
// direct evaluation p2_values at the Gauss point (the table the record replaces), in FP64 and with
// the record stored in FP32.  Built as a shared library by tests/test_face_basis_record.py.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dndsg_bodies.cuh"

using namespace dg;

template <class T>
static double record_error(const MeshView& m, const SetupParams& p, const std::vector<CellSetup>& cells) {
  const int64_t F = m.F;
  std::vector<double> faceW(6 * F), normal(2 * F), area(F), center(2 * F), w0(F);
  std::vector<T> basis(aos_size(F, kFaceBasisE));
  for (int64_t f = 0; f < F; f++)
    setup_face<T>(f, m, p, cells.data(), faceW.data(), normal.data(), area.data(), center.data(), w0.data(),
                  basis.data());
  double err = 0;
  for (int64_t f = 0; f < F; f++) {
    const FaceGeom g = face_geom(f, m);
    const int32_t L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
    const double sx = m.face_shift ? m.face_shift[2 * f] : 0.0, sy = m.face_shift ? m.face_shift[2 * f + 1] : 0.0;
    for (int side = 0; side < 2; side++) {
      const FaceBasisSide<T> rec(basis.data(), f, side);
      for (int q = 0; q < 3; q++) {
        double ref[5] = {0, 0, 0, 0, 0};
        if (side == 0) p2_values(cells[L].fr, g.gx[q], g.gy[q], ref);
        else if (R >= 0) p2_values(cells[R].fr, g.gx[q] - sx, g.gy[q] - sy, ref);
        T v[5];
        rec.at(q, v);
        for (int k = 0; k < 5; k++) err = std::max(err, std::fabs((double)v[k] - ref[k]));
      }
    }
  }
  return err;
}

extern "C" int face_basis_check(int64_t N, int64_t F, const double* node_xy, const int32_t* cell_nodes,
                                const int32_t* face_nodes, const int32_t* face_cells, const int32_t* face_bc,
                                const double* face_shift, int use_local_coord, double* err64, double* err32) {
  MeshView m{N, F, node_xy, cell_nodes, face_nodes, face_cells, face_bc, face_shift};
  SetupParams p{};
  p.use_local_coord = use_local_coord;
  p.weight_len_scale = 1.0;
  p.wall_weight = p.far_weight = p.tang_weight = p.tang_weight_mod_min = 1.0;
  std::vector<CellSetup> cells(N);
  for (int64_t i = 0; i < N; i++)
    if (!setup_cell(i, m, p, cells[i])) return 1;
  *err64 = record_error<double>(m, p, cells);
  *err32 = record_error<float>(m, p, cells);
  return 0;
}
