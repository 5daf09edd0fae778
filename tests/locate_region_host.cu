// Host build of the tile-shared point location (locate_region in
// sdtfe_b200/csrc/walk64.cuh) for tests/test_locate_region.py, which checks
// it against the oracle's location walk.  Test scaffolding only.
#include <vector>

#include "walk64.cuh"

using namespace sdtfe;

static std::vector<TriRec64> g_tri;

// triangles: corners (ax, ay, bx, by, cx, cy) and neighbours (n_CB, n_AC, n_BA, tet)
extern "C" void lr_set_triangles(const double* abc, const int* nb, int n) {
  g_tri.resize(n);
  for (int i = 0; i < n; ++i) {
    g_tri[i].a = make_double2(abc[6 * i + 0], abc[6 * i + 1]);
    g_tri[i].b = make_double2(abc[6 * i + 2], abc[6 * i + 3]);
    g_tri[i].c = make_double2(abc[6 * i + 4], abc[6 * i + 5]);
    g_tri[i].nb = make_int4(nb[4 * i + 0], nb[4 * i + 1], nb[4 * i + 2], nb[4 * i + 3]);
  }
}

extern "C" int lr_locate_region(double xlo, double xhi, double ylo, double yhi, int max_steps,
                                int* start, int* steps) {
  return locate_region(g_tri.data(), xlo, xhi, ylo, yhi, max_steps, start, steps);
}
