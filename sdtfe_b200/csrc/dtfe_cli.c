/* dtfe_cli.c - the `dtfe` program: the reference's example driver
 * (src/main.c:35-195) on this library.
 *
 *   dtfe [ path n_particles grid_dim center_x center_y center_z field_width
 *          field_depth particle_mass mc_box_width n_mc_samples sample_factor ]
 *
 * Same arguments, prompts for missing ones, and steps: read n_particles
 * float32 positions (x[n], y[n], z[n], the layout convert_to_qhdata reads),
 * shuffle for a sample_factor subsample, rotate by three rand() angles about
 * the field centre, triangulate, map (compute_density, on the GPU), and write
 * ./<file>.rho.bin (write_rho) and ./<file>.rho.tiff (write_image).
 *
 * Triangulation: this library has no Qhull of its own (triangulate() calls a
 * registered backend), so the program registers SciPy's Qhull through an
 * embedded Python interpreter - the interpreter found on PATH as python3, with
 * its environment's packages - and passes the reference's options.  A build
 * against a C Qhull would register that instead; nothing else changes.
 *
 * Beyond the reference: SDTFE_SEED=<n> replaces the time-of-day seed of
 * srand() (reproducible runs), and the library's SDTFE_PRECISION=mixed
 * selects the mixed-precision walk. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "dtfe.h"
#include "io.h"
#include "sdtfe_b200.h"
#include "triangulate.h"
#include "utils.h"

static PyObject *g_cells = NULL; /* cells(bytes, n, options) -> (simplices, neighbors, nt) */

static const char *kQhullPy =
    "import numpy as np\n"
    "from scipy.spatial import Delaunay\n"
    "def cells(buf, n, options):\n"
    "    pts = np.frombuffer(buf, dtype=np.float64).reshape(n, 4)[:, :3]\n"
    "    opts = ' '.join(o for o in options.split() if o not in ('qhull', 'd'))\n"
    "    d = Delaunay(np.ascontiguousarray(pts), qhull_options=opts)\n"
    "    s = np.ascontiguousarray(d.simplices, dtype=np.int32)\n"
    "    nb = np.ascontiguousarray(d.neighbors, dtype=np.int32)\n"
    "    return s.tobytes(), nb.tobytes(), len(s)\n";

static int scipy_cells(const double *xyz4, int n, const char *options, int **simplices,
                       int **neighbors, size_t *n_tetra, void *user) {
  (void)user;
  int rc = 1;
  PyObject *buf = PyBytes_FromStringAndSize((const char *)xyz4, (Py_ssize_t)n * 4 * sizeof(double));
  PyObject *res = buf ? PyObject_CallFunction(g_cells, "Ois", buf, n, options ? options : "") : NULL;
  char *s = NULL, *nb = NULL;
  Py_ssize_t ls = 0, lnb = 0;
  long long nt = 0;
  if (res && PyArg_ParseTuple(res, "y#y#L", &s, &ls, &nb, &lnb, &nt) && nt >= 0 &&
      ls == (Py_ssize_t)(nt * 4 * sizeof(int)) && lnb == ls) {
    *simplices = (int *)malloc((size_t)(ls ? ls : 1));
    *neighbors = (int *)malloc((size_t)(lnb ? lnb : 1));
    if (*simplices && *neighbors) {
      memcpy(*simplices, s, (size_t)ls);
      memcpy(*neighbors, nb, (size_t)lnb);
      *n_tetra = (size_t)nt;
      rc = 0;
    }
  }
  if (rc && PyErr_Occurred()) PyErr_Print();
  Py_XDECREF(res);
  Py_XDECREF(buf);
  return rc;
}

static int start_python(void) {
  PyConfig config;
  PyConfig_InitPythonConfig(&config);
  /* located on PATH, so that a virtual environment's packages are found */
  PyStatus st = PyConfig_SetBytesString(&config, &config.program_name, "python3");
  if (!PyStatus_Exception(st)) st = Py_InitializeFromConfig(&config);
  PyConfig_Clear(&config);
  if (PyStatus_Exception(st)) return 1;
  PyObject *globals = PyDict_New();
  if (!globals) return 1;
  PyDict_SetItemString(globals, "__builtins__", PyEval_GetBuiltins());
  PyObject *r = PyRun_String(kQhullPy, Py_file_input, globals, globals);
  if (!r) {
    PyErr_Print();
    Py_DECREF(globals);
    return 1;
  }
  Py_DECREF(r);
  g_cells = PyDict_GetItemString(globals, "cells");
  Py_XINCREF(g_cells);
  Py_DECREF(globals);
  return g_cells ? 0 : 1;
}

static const char *base_name(const char *path) {
  const char *s = strrchr(path, '/');
  return s ? s + 1 : path;
}

int main(int argc, char *argv[]) {
  char filename[512];
  if (argc < 2) {
    printf("Usage: dtfe [ path_to_file n_particles grid_dim center_x center_y center_z "
           "field_width field_depth particle_mass mc_box_width n_mc_samples sample_factor ]\n");
    printf("Enter the file location):\n");
    if (scanf("%511s", filename) != 1) return EXIT_FAILURE;
  } else {
    snprintf(filename, sizeof(filename), "%s", argv[1]);
  }
  long n_in = 0;
  int grid_dim = 0, n_mc_samples = 0;
  double center[3], box_len = 0, box_len_z = 0;
  float p_mass = 0, mc_box_width = 0, sample_factor = 0;
#define ASK(idx, prompt, fmt, ptr, conv)             \
  do {                                               \
    if (argc <= (idx)) {                             \
      printf(prompt);                                \
      if (scanf(fmt, ptr) != 1) return EXIT_FAILURE; \
    } else {                                         \
      *(ptr) = conv(argv[idx]);                      \
    }                                                \
  } while (0)
  ASK(2, "Enter the number of particles in the file:\n", "%ld", &n_in, atol);
  ASK(3, "Enter the grid cells per dimension (square assumed):\n", "%d", &grid_dim, atoi);
  if (argc < 7) {
    printf("Enter the center of the 3D field volume (use spaces to separate coordinates):\n");
    if (scanf("%lf%lf%lf", &center[0], &center[1], &center[2]) != 3) return EXIT_FAILURE;
  } else {
    for (int k = 0; k < 3; ++k) center[k] = atof(argv[4 + k]);
  }
  ASK(7, "Enter the width of the 2D field (square assumed):\n", "%lf", &box_len, atof);
  ASK(8, "Enter the depth of the 3D field (set limts of integration):\n", "%lf", &box_len_z, atof);
  ASK(9, "Enter the particle mass\n", "%f", &p_mass, (float)atof);
  ASK(10, "Enter the width for the Monte Carlo sample volume of each pixel:\n", "%f",
      &mc_box_width, (float)atof);
  ASK(11, "Enter number of Monte Carlo samples for each pixel:\n", "%d", &n_mc_samples, atoi);
  ASK(12, "Enter the subsample factor:\n", "%f", &sample_factor, (float)atof);
#undef ASK
  if (n_in <= 0 || grid_dim <= 0 || n_mc_samples <= 0 || !(sample_factor > 0)) {
    fprintf(stderr, "dtfe: n_particles, grid_dim, n_mc_samples and sample_factor must be > 0\n");
    return EXIT_FAILURE;
  }
  const size_t n_particles = (size_t)n_in;

  const char *env_seed = getenv("SDTFE_SEED");
  const unsigned int seed =
      env_seed ? (unsigned int)strtoul(env_seed, NULL, 10) : (unsigned int)time(NULL);
  srand(seed);
  printf("Using prng seed: %u\n", seed);
  p_mass = p_mass / sample_factor;

  float *buff = (float *)malloc(n_particles * sizeof(float) * 3);
  FILE *f = fopen(filename, "rb");
  if (!buff || !f) {
    fprintf(stderr, "dtfe: cannot read %s\n", filename);
    return EXIT_FAILURE;
  }
  const size_t got = fread(buff, sizeof(float), n_particles * 3, f);
  fclose(f);
  if (got != n_particles * 3) {
    fprintf(stderr, "dtfe: %s holds %zu floats, expected %zu\n", filename, got, n_particles * 3);
    return EXIT_FAILURE;
  }

  printf("Converting to Qhull format...\n");
  double *particle_data = convert_to_qhdata(buff, n_particles);
  printf("Shuffling the data...\n");
  const size_t n_shuffle = (size_t)(n_particles * sample_factor);
  if (n_shuffle < 5) {
    fprintf(stderr, "dtfe: not enough particles\n");
    return EXIT_FAILURE;
  }
  shuffle_buff(particle_data, (int)n_particles, (int)n_shuffle);
  double theta[3];
  for (int k = 0; k < 3; ++k) theta[k] = (double)rand() / RAND_MAX * 2.0 * M_PI;
  printf("Rotating with theta=[%lf %lf %lf]...\n", theta[0], theta[1], theta[2]);
  rotate3d(particle_data, n_shuffle, theta, center);

  printf("Creating Delaunay triangulation...\n");
  if (start_python() != 0) {
    fprintf(stderr, "dtfe: could not start the Python interpreter for SciPy's Qhull\n");
    return EXIT_FAILURE;
  }
  dtfe_set_triangulator(scipy_cells, NULL);
  size_t n_tetra = 0;
  int *tetra_data = triangulate(particle_data, (int)n_shuffle, &n_tetra, "qhull d Qz Qt Qbb");
  if (!tetra_data) return EXIT_FAILURE;
  printf("Done creating %zu tetrahedra.\n", n_tetra);

  printf("Creating %dx%d surface density field...\n", grid_dim, grid_dim);
  printf("Center: %f, %f, %f\n", center[0], center[1], center[2]);
  printf("box_len:%f box_len_z: %f\n", box_len, box_len_z);
  double *rho = (double *)calloc((size_t)grid_dim * grid_dim, sizeof(double));
  if (!rho) return EXIT_FAILURE;
  dtfe_clear_error();
  compute_density(particle_data, (int)n_shuffle, tetra_data, (int)n_tetra, grid_dim, box_len,
                  box_len_z, rho, p_mass, center[0], center[1], center[2], n_mc_samples,
                  mc_box_width);
  const int failed = dtfe_last_error()[0] != '\0';
  free(tetra_data);
  free(particle_data);
  if (failed) return EXIT_FAILURE; /* compute_density reported the failure */

  char output[1024], image[1024];
  snprintf(output, sizeof(output), "./%s.rho.bin", base_name(filename));
  snprintf(image, sizeof(image), "./%s.rho.tiff", base_name(filename));
  write_image(image, rho, grid_dim);
  write_rho(output, &rho, grid_dim * grid_dim);
  free(rho);
  free(buff);
  Py_XDECREF(g_cells);
  Py_FinalizeEx();
  return EXIT_SUCCESS;
}
