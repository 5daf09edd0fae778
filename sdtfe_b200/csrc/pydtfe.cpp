// pydtfe.cpp - the reference's Python module (python/pydtfe.cpp:205-384) over
// this library's C ABI: same module name, functions, argument names, defaults,
// dtypes and errors.  Each call prepares the particles on the host
// (convert_to_qhdata, shuffle_buff, rotate3d), triangulates them with the host
// Qhull (SciPy's, registered below as the triangulate() backend), and hands
// them to the drop-in entry points, whose work runs on the GPU.  Unlike the
// reference, the GIL is released while the GPU works.
//
// Additions beyond the reference's module: set_seed(), set_precision(),
// kernel_launches().
//
// The module does not link the library by name: it dlopens its sibling
// libsdtfe_b200.so by path and resolves every entry point through that
// handle.  The drop-in names (compute_density, shuffle_buff, ...) are also the
// reference's, so a process that has the reference's libdtfe loaded globally
// would otherwise bind this module to the reference's CPU code.
#include <dlfcn.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cstdlib>
#include <cstring>
#include <optional>
#include <string>

extern "C" {
#include "dtfe.h"
#include "sdtfe_b200.h"
#include "triangulate.h"
#include "utils.h"
}

namespace py = pybind11;

namespace {

// entry points of libsdtfe_b200.so, resolved in that library only
struct Api {
  decltype(&::convert_to_qhdata) convert_to_qhdata;
  decltype(&::shuffle_buff) shuffle_buff;
  decltype(&::rotate3d) rotate3d;
  decltype(&::triangulate) triangulate;
  decltype(&::compute_density) compute_density;
  decltype(&::compute_3d_density) compute_3d_density;
  decltype(&::interpolate_to_3d_grid) interpolate_to_3d_grid;
  decltype(&::pre_compute_vol) pre_compute_vol;
  decltype(&::dtfe_set_triangulator) dtfe_set_triangulator;
  decltype(&::dtfe_set_seed) dtfe_set_seed;
  decltype(&::dtfe_set_default_precision) dtfe_set_default_precision;
  decltype(&::dtfe_last_error) dtfe_last_error;
  decltype(&::dtfe_clear_error) dtfe_clear_error;
  decltype(&::dtfe_kernel_launches) dtfe_kernel_launches;
};
Api api;

void load_api() {
  Dl_info info;
  if (!dladdr(reinterpret_cast<void*>(&load_api), &info) || !info.dli_fname)
    throw std::runtime_error("pydtfe: cannot locate its own module file");
  std::string dir = info.dli_fname;
  dir = dir.substr(0, dir.find_last_of('/'));  // .../sdtfe_b200/pydtfe
  const std::string path = dir.substr(0, dir.find_last_of('/')) + "/libsdtfe_b200.so";
  void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
  if (!h) throw std::runtime_error(std::string("pydtfe: cannot load ") + path + ": " + dlerror());
  auto get = [&](auto& fn, const char* name) {
    void* p = dlsym(h, name);
    if (!p) throw std::runtime_error(std::string("pydtfe: ") + path + " lacks " + name);
    fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(p);
  };
  get(api.convert_to_qhdata, "convert_to_qhdata");
  get(api.shuffle_buff, "shuffle_buff");
  get(api.rotate3d, "rotate3d");
  get(api.triangulate, "triangulate");
  get(api.compute_density, "compute_density");
  get(api.compute_3d_density, "compute_3d_density");
  get(api.interpolate_to_3d_grid, "interpolate_to_3d_grid");
  get(api.pre_compute_vol, "pre_compute_vol");
  get(api.dtfe_set_triangulator, "dtfe_set_triangulator");
  get(api.dtfe_set_seed, "dtfe_set_seed");
  get(api.dtfe_set_default_precision, "dtfe_set_default_precision");
  get(api.dtfe_last_error, "dtfe_last_error");
  get(api.dtfe_clear_error, "dtfe_clear_error");
  get(api.dtfe_kernel_launches, "dtfe_kernel_launches");
}

// triangulate() backend: Qhull through scipy.spatial.Delaunay with the options
// the caller passes (the reference passes "qhull d Qz Qt Qbb"; SciPy adds "d").
int scipy_qhull(const double* xyz4, int n, const char* options, int** simplices, int** neighbors,
                size_t* n_tetra, void*) {
  py::gil_scoped_acquire gil;
  try {
    std::string opts = options ? options : "";
    for (const char* drop : {"qhull ", "d "}) {
      const size_t p = opts.find(drop);
      if (p != std::string::npos) opts.erase(p, std::strlen(drop));
    }
    py::array_t<double> pts({(py::ssize_t)n, (py::ssize_t)3});
    auto w = pts.mutable_unchecked<2>();
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) w(i, k) = xyz4[4 * (size_t)i + k];
    py::object tri = py::module_::import("scipy.spatial")
                         .attr("Delaunay")(pts, py::arg("qhull_options") = opts);
    auto s = py::array_t<int, py::array::c_style | py::array::forcecast>(tri.attr("simplices"));
    auto nb = py::array_t<int, py::array::c_style | py::array::forcecast>(tri.attr("neighbors"));
    const size_t nt = (size_t)s.shape(0);
    *simplices = (int*)malloc(sizeof(int) * 4 * (nt ? nt : 1));
    *neighbors = (int*)malloc(sizeof(int) * 4 * (nt ? nt : 1));
    if (!*simplices || !*neighbors) return 1;
    std::memcpy(*simplices, s.data(), sizeof(int) * 4 * nt);
    std::memcpy(*neighbors, nb.data(), sizeof(int) * 4 * nt);
    *n_tetra = nt;
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

using fpos = py::array_t<float, py::array::f_style | py::array::forcecast>;

struct Prepared {
  double* data = nullptr;
  size_t n = 0;
  int* tetra = nullptr;
  size_t nt = 0;
  ~Prepared() {
    free(tetra);
    free(data);
  }
};

void check_shape(const fpos& pos) {
  if (pos.ndim() != 2 || pos.shape(1) != 3)
    throw py::value_error("incorrect shape of particle position array");
}

void triangulate_into(Prepared& P) {
  api.dtfe_clear_error();
  P.tetra = api.triangulate(P.data, (int)P.n, &P.nt, "qhull d Qz Qt Qbb");
  if (!P.tetra) throw std::runtime_error(std::string("triangulation failed: ") + api.dtfe_last_error());
}

// the drop-ins return void and report failures through dtfe_last_error
void raise_if_failed(const char* what) {
  const char* e = api.dtfe_last_error();
  if (e && *e) throw std::runtime_error(std::string(what) + ": " + e);
}

// python/pydtfe.cpp:16-66
py::array_t<double> compute_density_py(fpos particle_pos, std::array<double, 3> center,
                                       unsigned grid_dim, float sample_factor, double box_width,
                                       double box_depth, double particle_mass, double mc_box_width,
                                       unsigned mc_sample_count,
                                       std::optional<std::array<double, 3>> rotation_angle) {
  check_shape(particle_pos);
  Prepared P;
  const size_t n_particles = particle_pos.shape(0);
  P.data = api.convert_to_qhdata(particle_pos.data(), n_particles);
  const size_t n_shuffle = n_particles * sample_factor;
  if (n_shuffle < 5) throw py::value_error("not enough particles");
  api.shuffle_buff(P.data, (int)n_particles, (int)n_shuffle);
  particle_mass /= sample_factor;
  if (rotation_angle) api.rotate3d(P.data, n_shuffle, rotation_angle->data(), center.data());
  P.n = n_shuffle;
  triangulate_into(P);
  py::array_t<double> rho({(py::ssize_t)grid_dim, (py::ssize_t)grid_dim});
  std::fill(rho.mutable_data(), rho.mutable_data() + (size_t)grid_dim * grid_dim, 0.);
  api.dtfe_clear_error();
  {
    py::gil_scoped_release nogil;
    api.compute_density(P.data, (int)P.n, P.tetra, (int)P.nt, (int)grid_dim, box_width, box_depth,
                    rho.mutable_data(), (float)particle_mass, center[0], center[1], center[2],
                    (int)mc_sample_count, mc_box_width);
  }
  raise_if_failed("compute_surface_density");
  return rho;
}

// python/pydtfe.cpp:68-112
py::array_t<double> compute_3d_density_py(fpos particle_pos, std::array<double, 3> center,
                                          unsigned grid_dim, float sample_factor,
                                          double box_length, double particle_mass,
                                          unsigned supersampling) {
  check_shape(particle_pos);
  Prepared P;
  const size_t n_particles = particle_pos.shape(0);
  P.data = api.convert_to_qhdata(particle_pos.data(), n_particles);
  const size_t n_shuffle = n_particles * sample_factor;
  if (n_shuffle < 5) throw py::value_error("not enough particles");
  api.shuffle_buff(P.data, (int)n_particles, (int)n_shuffle);
  particle_mass /= sample_factor;
  P.n = n_shuffle;
  triangulate_into(P);
  const size_t g = grid_dim;
  py::array_t<double> rho({(py::ssize_t)g, (py::ssize_t)g, (py::ssize_t)g});
  std::fill(rho.mutable_data(), rho.mutable_data() + g * g * g, 0.);
  api.dtfe_clear_error();
  {
    py::gil_scoped_release nogil;
    api.compute_3d_density(P.data, (int)P.n, P.tetra, (int)P.nt, (int)grid_dim, box_length,
                       rho.mutable_data(), (float)particle_mass, center[0], center[1], center[2],
                       supersampling);
  }
  raise_if_failed("compute_3d_density");
  return rho;
}

// python/pydtfe.cpp:114-171
py::array_t<double> interpolate_field2grid(fpos particle_pos, py::array_t<float> particle_value,
                                           std::array<double, 3> center, unsigned grid_dim,
                                           float sample_factor, double box_length,
                                           unsigned supersampling) {
  check_shape(particle_pos);
  const size_t n_particles = particle_pos.shape(0);
  if (particle_value.ndim() < 1 || (size_t)particle_value.shape(0) != n_particles)
    throw py::value_error("different length of particle position and value arrays");
  Prepared P;
  P.data = api.convert_to_qhdata(particle_pos.data(), n_particles);
  if (sample_factor != 1.0f)
    throw py::value_error("`sample_factor != 1.0f` not supported at the moment");
  P.n = n_particles;
  triangulate_into(P);
  auto val = particle_value.unchecked<1>();
  for (size_t i = 0; i < n_particles; ++i) P.data[4 * i + 3] = val(i);
  const size_t g = grid_dim;
  py::array_t<double> grid({(py::ssize_t)g, (py::ssize_t)g, (py::ssize_t)g});
  std::fill(grid.mutable_data(), grid.mutable_data() + g * g * g, 0.);
  api.dtfe_clear_error();
  {
    py::gil_scoped_release nogil;
    api.interpolate_to_3d_grid(P.data, (int)P.n, P.tetra, (int)P.nt, (int)grid_dim, box_length,
                           grid.mutable_data(), center[0], center[1], center[2], supersampling);
  }
  raise_if_failed("interpolate_field2grid");
  return grid;
}

// python/pydtfe.cpp:173-203
py::array_t<float> compute_particle_density_py(fpos particle_pos, double particle_mass) {
  check_shape(particle_pos);
  Prepared P;
  const size_t n_particles = particle_pos.shape(0);
  P.data = api.convert_to_qhdata(particle_pos.data(), n_particles);
  P.n = n_particles;
  triangulate_into(P);
  api.dtfe_clear_error();
  {
    py::gil_scoped_release nogil;
    api.pre_compute_vol(&P.data, (int)P.n, P.tetra, (int)P.nt, (float)particle_mass);
  }
  raise_if_failed("compute_particle_density");
  py::array_t<float> rho((py::ssize_t)n_particles);
  for (size_t i = 0; i < n_particles; ++i) rho.mutable_data()[i] = (float)P.data[4 * i + 3];
  return rho;
}

}  // namespace

PYBIND11_MODULE(_pydtfe, m) {
  m.doc() = "python interface to SDTFE (B200 GPU implementation)";
  load_api();
  api.dtfe_set_triangulator(scipy_qhull, nullptr);
  m.def("compute_surface_density", &compute_density_py,
        "surface density of a particle distribution from its DTFE (python/pydtfe.cpp:207)",
        py::arg("particle_pos"), py::arg("center"), py::arg("grid_dim"), py::arg("sample_factor"),
        py::arg("box_width"), py::arg("box_depth"), py::arg("particle_mass"),
        py::arg("mc_box_width"), py::arg("mc_sample_count"), py::arg("rotation_angle") = nullptr);
  m.def("compute_3d_density", &compute_3d_density_py,
        "volumetric DTFE density on a cube grid (python/pydtfe.cpp:263)", py::arg("particle_pos"),
        py::arg("center"), py::arg("grid_dim"), py::arg("sample_factor"), py::arg("box_length"),
        py::arg("particle_mass"), py::arg("supersampling") = 1u);
  m.def("interpolate_field2grid", &interpolate_field2grid,
        "DTFE interpolation of a particle field to a cube grid (python/pydtfe.cpp:311)",
        py::arg("particle_pos"), py::arg("particle_value"), py::arg("center"),
        py::arg("grid_dim"), py::arg("sample_factor"), py::arg("box_length"),
        py::arg("supersampling") = 1u);
  m.def("compute_particle_density", &compute_particle_density_py,
        "DTFE density at the particle positions (python/pydtfe.cpp:364)",
        py::arg("particle_pos"), py::arg("particle_mass"));
  m.def("set_seed", [](uint64_t s) { api.dtfe_set_seed(s); },
        "fix the Monte Carlo sample key (0: one rand() draw per call)", py::arg("seed"));
  m.def("kernel_launches", []() { return api.dtfe_kernel_launches(); },
        "CUDA kernels the library has launched in this process");
  m.def("set_precision", [](const std::string& p) {
    if (p == "fp64") api.dtfe_set_default_precision(DTFE_FP64);
    else if (p == "mixed") api.dtfe_set_default_precision(DTFE_MIXED);
    else throw py::value_error("precision must be 'fp64' or 'mixed'");
  }, "walk arithmetic of the drop-in calls", py::arg("precision"));
}
