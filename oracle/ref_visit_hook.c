/*
 * ref_visit_hook.c - records which tetrahedra the reference walk visits.
 *
 * TEST INFRASTRUCTURE ONLY.  Built into oracle/_ref/libdtfe_refhook.so and
 * loaded with RTLD_GLOBAL before libdtfe_refh.so.  The reference's walk calls
 * its exported rayTetraPlucker_full (src/dtfe.c:29) through the PLT (the
 * sources are built -fPIC with default semantic interposition), so the call
 * binds to the definition below, which logs the four vertex-array offsets of
 * the tet (they identify the tet row) and forwards to the reference's own
 * function, whose address the loader passes in with refhook_set_real (a
 * lookup through the harness library's own handle, which resolves to the
 * harness's definition rather than this one).  Repeated calls for the same tet
 * (the perturbation retries of src/dtfe.c:330-349) are logged as well; the
 * caller folds consecutive duplicates.
 */
#include <stddef.h>

typedef int (*rtp_fn)(double *, double **, int *, int *, double *, double *, int *);

static rtp_fn real_fn;
static const double *log_base;   /* particle_data of the traced mesh */
static int *log_buf;             /* 4 vertex ids per logged call      */
static long log_cap, log_len;    /* in calls                          */
static int *log_ray_start;       /* first call index of each ray      */
static int log_nrays;

void refhook_set_real(void *fn) { real_fn = (rtp_fn)fn; }

void refhook_begin(const double *base, int *buf, long cap, int *ray_start, int n_rays) {
  log_base = base;
  log_buf = buf;
  log_cap = cap;
  log_len = 0;
  log_ray_start = ray_start;
  log_nrays = n_rays;
}

/* called by the harness before each ray */
void refhook_ray(int i) {
  if (log_ray_start && i < log_nrays) log_ray_start[i] = (int)log_len;
}

long refhook_end(void) {
  long n = log_len;
  log_buf = NULL;
  log_ray_start = NULL;
  return n;
}

int rayTetraPlucker_full(double plRay2[], double *vert[], int *enterFace, int *leaveFace,
                         double enterPoint[], double leavePoint[], int *isSpecialCase) {
  if (log_buf && log_len < log_cap) {
    for (int k = 0; k < 4; ++k) log_buf[log_len * 4 + k] = (int)((vert[k] - log_base) / 4);
    ++log_len;
  }
  return real_fn(plRay2, vert, enterFace, leaveFace, enterPoint, leavePoint, isSpecialCase);
}
