// Harness around the reference's own CPU path (setup_mlfma.cpp, integrate.cpp,
// solve.cpp, bicgs.cpp, compiled unmodified from the reference tree by
// oracle/Makefile); compiled with REF_GPU, around the reference's GPU path
// instead (gpu.cu, kernels.cu, matvec_gpu.cu, bicgs_gpu.cu: the same entry
// points, FP64 on the GPU).  TEST INFRASTRUCTURE ONLY: it is the checker used to pin
// the restated oracle (isg_oracle.c) and to produce the golden fixtures, and
// the CPU baseline arm of bench.py.  Nothing in the product links it.
//
// It defines the globals that the reference's driver owns (mom.cpp:4-69) and
// exposes a C entry point per reference routine.  Complex arrays are passed as
// interleaved (re, im) doubles, in the reference's tree order.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>
#include <omp.h>
#include "mpi.h"

using std::complex;

// ---- globals owned by the reference driver (mom.cpp:4-69) ----
double res = 0.1;
int box = 8;
int level = 5;
double k0 = 2 * M_PI;
int numunk = 0;
int numrx = 32;
double toli = 1e-5;
int iti = 300;
complex<double> *pos = nullptr;
int *unkmap = nullptr;
MPI_Comm MPI_COMM_MLFMA = 0;
double bicgst = 0, innert = 0, outert = 0;
int matvecin = 0, matvecout = 0;

// ---- reference routines (vars.h:14-38, bicgs.cpp) ----
void setup_mlfma();
void setup_bicgs();
#ifdef REF_GPU
void setup_gpu();  // gpu.cu:69, between the two as in mom.cpp:184-190
#endif
void mlfma(complex<double> *, complex<double> *);
void mlfmah(complex<double> *, complex<double> *);
void aggregate(complex<double> *, complex<double> *);
void aggregateh(complex<double> *, complex<double> *);
void bicgs(complex<double> *, complex<double> *, complex<double> *, bool);
complex<double> integrate(complex<double>, complex<double>);

// ---- reference tables (setup_mlfma.cpp:6-46) ----
extern int ninter;
extern int *numclus, *numsamp, *numterm;
extern double *clusize;
extern complex<double> **clusc;
extern int **clusnear, **clusfar, **traid;
extern complex<double> *near, *coeff_multi, *basis_local;
extern double **interp, **anterp;
extern int **intind, **antind;
extern complex<double> **shiftmul, **shiftloc, **trans;
extern double *interph, *anterph;
extern int *intindh, *antindh;

static int g_ready_level = -1;
static double g_ready_k0 = 0;
static int g_ready_numrx = -1;

// Runs fn with stdout sent to a temporary file; returns what was printed.
template <class F>
static std::string capture_stdout(F fn) {
  fflush(stdout);
  char path[] = "/tmp/isgref_outXXXXXX";
  int fd = mkstemp(path);
  int saved = dup(1);
  dup2(fd, 1);
  fn();
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  std::string out;
  lseek(fd, 0, SEEK_SET);
  char buf[4096];
  ssize_t n;
  while ((n = read(fd, buf, sizeof buf)) > 0) out.append(buf, (size_t)n);
  close(fd);
  unlink(path);
  return out;
}

extern "C" {

// Builds the reference's MLFMA tables for a grid of box*2^(lvl-1) pixels per
// side.  setup_mlfma.cpp:286 reads the one-rank pair schedule from the working
// directory, so the call runs inside a scratch directory holding it.
int ref_setup(int lvl, double wavenumber, int nrx) {
  if (lvl == g_ready_level && wavenumber == g_ready_k0 && nrx == g_ready_numrx) return 0;
  level = lvl;
  k0 = wavenumber;
  numrx = nrx;
  double dim = res * box * std::pow(2.0, level - 1);
  numunk = (int)std::pow(dim / res, 2);
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) return -1;
  char dir[] = "/tmp/isgref_XXXXXX";
  if (!mkdtemp(dir)) return -2;
  std::string sched = std::string(dir) + "/internodes001.dat";
  FILE *f = fopen(sched.c_str(), "w");
  if (!f) return -3;
  fprintf(f, "0\n");
  fclose(f);
  if (chdir(dir) != 0) return -4;
  capture_stdout([] {
    setup_mlfma();
#ifdef REF_GPU
    setup_gpu();
#endif
    setup_bicgs();
  });
  if (chdir(cwd) != 0) return -5;
  unlink(sched.c_str());
  rmdir(dir);
  g_ready_level = lvl;
  g_ready_k0 = wavenumber;
  g_ready_numrx = nrx;
  return 0;
}

int ref_numunk(void) { return numunk; }
int ref_level(void) { return level; }
int ref_numsamp(int i) { return numsamp[i]; }
int ref_numterm(int i) { return numterm[i]; }
int ref_ninter(void) { return ninter; }
int ref_omp_threads(void) { return omp_get_max_threads(); }

void ref_mlfma(double *x, double *r) { mlfma((complex<double> *)x, (complex<double> *)r); }
void ref_mlfmah(double *x, double *r) { mlfmah((complex<double> *)x, (complex<double> *)r); }
void ref_aggregate(double *x, double *rx) { aggregate((complex<double> *)x, (complex<double> *)rx); }
void ref_aggregateh(double *x, double *rx) { aggregateh((complex<double> *)x, (complex<double> *)rx); }

// bicgs(x, g, b, hermitian) with the given tolerance and iteration cap.
// Returns the iteration count that bicgs.cpp:176 prints, or -1.
int ref_bicgs(double *x, double *g, double *b, int hermitian, double tol, int maxit) {
  toli = tol;
  iti = maxit;
  std::string out = capture_stdout([&] {
    bicgs((complex<double> *)x, (complex<double> *)g, (complex<double> *)b, hermitian != 0);
  });
  int h = 0, it = -1, mv = 0;
  size_t at = out.rfind("NUMBER OF");
  if (at != std::string::npos) sscanf(out.c_str() + at, "NUMBER OF %d ITERATIONS: %d (%d)", &h, &it, &mv);
  return it;
}

void ref_integrate(double tx, double ty, double bx, double by, double *out) {
  complex<double> v = integrate(complex<double>(tx, ty), complex<double>(bx, by));
  out[0] = v.real();
  out[1] = v.imag();
}

// Raw views of the reference's tables; `lvl` selects the per-level array.
const void *ref_table(const char *name, int lvl) {
  std::string n(name);
  if (n == "numclus") return numclus;
  if (n == "numsamp") return numsamp;
  if (n == "clusize") return clusize;
  if (n == "clusc") return clusc[lvl];
  if (n == "clusnear") return clusnear[lvl];
  if (n == "clusfar") return clusfar[lvl];
  if (n == "traid") return traid[lvl];
  if (n == "near") return near;
  if (n == "coeff_multi") return coeff_multi;
  if (n == "basis_local") return basis_local;
  if (n == "interp") return interp[lvl];
  if (n == "anterp") return anterp[lvl];
  if (n == "intind") return intind[lvl];
  if (n == "antind") return antind[lvl];
  if (n == "shiftmul") return shiftmul[lvl];
  if (n == "shiftloc") return shiftloc[lvl];
  if (n == "trans") return trans[lvl];
  if (n == "interph") return interph;
  if (n == "anterph") return anterph;
  if (n == "intindh") return intindh;
  if (n == "antindh") return antindh;
  if (n == "pos") return pos;
  if (n == "unkmap") return unkmap;
  return nullptr;
}

}  // extern "C"
