// libcvcb200_tmlqcd.so: the tmLQCD library-wrapper ABI (tmLQCD.h:33-58 of the
// reference) over the B200 solver, for programs that take their propagators
// from tmLQCD (cvc_exact2_xspace.c:131-150,206-216,436-547, p2gg_xspace.c:
// 139-158,434-585).
//
// Input file (tmLQCD style, "Key = value", keys case-insensitive, '#'
// comments), read by tmLQCD_invert_init:
//   L, LX, LY, LZ, T                lattice extents (L sets all three spatial)
//   InitialStoreCounter             nstore (default 0)
//   Measurements                    nsave (default 1)
//   GaugeConfigInputFile            gauge file prefix (default "conf")
//   kappa, 2KappaMu                 defaults for the operators
//   ThetaT, ThetaX, ThetaY, ThetaZ  boundary phases in units of pi/L
//                                   (default 1, 0, 0, 0: antiperiodic in time,
//                                   as CVC's BCangle)
//   SolverPrecision                 squared residual |b - D x|^2 (default 1e-20);
//                                   absolute, as in tmLQCD, unless
//   UseRelativePrecision            is yes: then relative to |b|^2 (default no)
//   MaxSolverIterations             (default 20000)
//   PropagatorFilePrefix            for write_prop (default "source")
//   GPUDevice                       CUDA device (default 0)
//   GPUPrecision                    inner iterations: single (default), half
//                                   or double; FP64 reliable updates always
//   BeginOperator <name> ... EndOperator   one operator per block, with its
//                                   own kappa, 2KappaMu, SolverPrecision,
//                                   MaxSolverIterations; without blocks, one
//                                   operator from the defaults.
// Normalisation: tmLQCD's D = 2 kappa Q, so the returned propagator is
// Q^-1 source / (2 kappa) with Q the operator of Q_phi_tbc.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cvcb.h"
#include "../../include/cvcb_tmlqcd.h"

namespace {

struct Operator {
  double kappa = 0.125, two_kappa_mu = 0.0, precision = 1e-20;
  int max_iter = 20000;
  bool relative = false;  // SolverPrecision relative to |b|^2 (tmLQCD: absolute)
};

struct State {
  bool init = false;
  int verbose = 0;
  int T = 0, LX = 0, LY = 0, LZ = 0;
  int nstore = 0, nsave = 1, device = 0, gpu_precision = CVCB_PREC_SINGLE;
  double theta[4] = {1.0, 0.0, 0.0, 0.0};
  std::string gauge_prefix = "conf", prop_prefix = "source";
  std::vector<Operator> ops;
  std::vector<double> gauge;
  cvcb_lattice *lat = nullptr;
  int nwritten = 0;
};
State g;

std::string lower(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

bool set_op_key(Operator &op, const std::string &k, const std::string &v) {
  if (k == "kappa") op.kappa = std::atof(v.c_str());
  else if (k == "2kappamu") op.two_kappa_mu = std::atof(v.c_str());
  else if (k == "solverprecision") op.precision = std::atof(v.c_str());
  else if (k == "maxsolveriterations") op.max_iter = std::atoi(v.c_str());
  else if (k == "userelativeprecision") op.relative = lower(trim(v)) == "yes";
  else return false;
  return true;
}

int read_input(const char *name) {
  FILE *f = std::fopen(name, "r");
  if (!f) {
    std::fprintf(stderr, "[tmLQCD_invert_init] cannot open input file %s\n", name);
    return 1;
  }
  Operator defaults;
  std::vector<std::pair<std::string, std::string>> block;
  bool in_block = false;
  std::vector<std::vector<std::pair<std::string, std::string>>> blocks;
  char line[1024];
  while (std::fgets(line, sizeof line, f)) {
    std::string s = line;
    const size_t hash = s.find('#');
    if (hash != std::string::npos) s.resize(hash);
    s = trim(s);
    if (s.empty()) continue;
    const std::string ls = lower(s);
    if (ls.rfind("beginoperator", 0) == 0) {
      in_block = true;
      block.clear();
      continue;
    }
    if (ls.rfind("endoperator", 0) == 0) {
      in_block = false;
      blocks.push_back(block);
      continue;
    }
    const size_t eq = s.find('=');
    if (eq == std::string::npos) continue;
    const std::string k = lower(trim(s.substr(0, eq))), v = trim(s.substr(eq + 1));
    if (in_block) {
      block.emplace_back(k, v);
      continue;
    }
    if (set_op_key(defaults, k, v)) continue;
    if (k == "l") g.LX = g.LY = g.LZ = std::atoi(v.c_str());
    else if (k == "lx") g.LX = std::atoi(v.c_str());
    else if (k == "ly") g.LY = std::atoi(v.c_str());
    else if (k == "lz") g.LZ = std::atoi(v.c_str());
    else if (k == "t") g.T = std::atoi(v.c_str());
    else if (k == "initialstorecounter") g.nstore = std::atoi(v.c_str());
    else if (k == "measurements") g.nsave = std::atoi(v.c_str());
    else if (k == "gaugeconfiginputfile") g.gauge_prefix = v;
    else if (k == "propagatorfileprefix") g.prop_prefix = v;
    else if (k == "thetat") g.theta[0] = std::atof(v.c_str());
    else if (k == "thetax") g.theta[1] = std::atof(v.c_str());
    else if (k == "thetay") g.theta[2] = std::atof(v.c_str());
    else if (k == "thetaz") g.theta[3] = std::atof(v.c_str());
    else if (k == "gpudevice") g.device = std::atoi(v.c_str());
    else if (k == "gpuprecision") {
      const std::string lv = lower(v);
      g.gpu_precision = lv == "double" ? CVCB_PREC_DOUBLE
                        : lv == "half" ? CVCB_PREC_HALF : CVCB_PREC_SINGLE;
    }
  }
  std::fclose(f);
  if (in_block) {
    std::fprintf(stderr, "[tmLQCD_invert_init] BeginOperator without EndOperator in %s\n", name);
    return 2;
  }
  g.ops.clear();
  for (const auto &b : blocks) {
    Operator op = defaults;
    for (const auto &kv : b) set_op_key(op, kv.first, kv.second);
    g.ops.push_back(op);
  }
  if (g.ops.empty()) g.ops.push_back(defaults);
  if (g.T <= 0 || g.LX <= 0 || g.LY <= 0 || g.LZ <= 0) {
    std::fprintf(stderr, "[tmLQCD_invert_init] T and L must be set in %s\n", name);
    return 2;
  }
  return 0;
}

}  // namespace

extern "C" {

int tmLQCD_invert_init(int argc, char *argv[], const int verbose) {
  if (g.init) tmLQCD_finalise();
  g = State();
  g.verbose = verbose;
  const char *input = "invert.input";
  for (int i = 1; i + 1 < argc; ++i)
    if (std::strcmp(argv[i], "-f") == 0) input = argv[i + 1];
  if (read_input(input)) return 1;
  if (cvcb_lattice_create(&g.lat, g.T, g.LX, g.LY, g.LZ, g.device) != CVCB_OK) {
    std::fprintf(stderr, "[tmLQCD_invert_init] %s\n", cvcb_last_error());
    return 3;
  }
  g.gauge.assign((size_t)72 * g.T * g.LX * g.LY * g.LZ, 0.0);
  g.init = true;
  if (verbose)
    std::printf("# [tmLQCD_invert_init] %dx%dx%dx%d, %zu operator(s), GPU %d\n", g.T, g.LX, g.LY,
                g.LZ, g.ops.size(), g.device);
  return 0;
}

int tmLQCD_read_gauge(const int nconfig) {
  if (!g.init) return 1;
  char name[1024];
  std::snprintf(name, sizeof name, "%s.%.4d", g.gauge_prefix.c_str(), nconfig);
  uint32_t sums[2];
  if (cvcb_read_lime_gauge_field_doubleprec(name, g.gauge.data(), g.T, g.LX, g.LY, g.LZ, sums) !=
      CVCB_OK) {
    std::fprintf(stderr, "[tmLQCD_read_gauge] %s\n", cvcb_last_error());
    return 2;
  }
  if (cvcb_upload_gauge(g.lat, g.gauge.data()) != CVCB_OK) {
    std::fprintf(stderr, "[tmLQCD_read_gauge] %s\n", cvcb_last_error());
    return 3;
  }
  if (g.verbose) {
    double plaq = 0, ls[2];
    cvcb_plaquette(g.lat, &plaq, ls);
    std::printf("# [tmLQCD_read_gauge] %s: checksum %#x %#x, plaquette %.16e\n", name, sums[0],
                sums[1], plaq);
  }
  return 0;
}

int tmLQCD_invert(double *const propagator, double *const source, const int op_id,
                  const int write_prop) {
  if (!g.init) return 1;
  if (!propagator || !source) return 2;
  if (op_id < 0 || op_id >= (int)g.ops.size()) return 3;
  const Operator &op = g.ops[op_id];
  const double mu = op.two_kappa_mu / (2.0 * op.kappa);
  if (cvcb_set_params(g.lat, op.kappa, mu, g.theta) != CVCB_OK) return 4;
  cvcb_solver_params p;
  cvcb_solver_defaults(&p);
  p.precision = g.gpu_precision;
  p.link_recon = g.gpu_precision == CVCB_PREC_DOUBLE ? 18 : 12;
  // the batched solver stops on |b - Q x| / |b|; tmLQCD's D x' = b with
  // x' = x / (2 kappa) has the same residual b - Q x
  double rel2 = op.precision;
  if (!op.relative) {  // absolute: |b - Q x|^2 <= precision
    const size_t nb = (size_t)24 * g.T * g.LX * g.LY * g.LZ;
    double b2 = 0.0;
    for (size_t i = 0; i < nb; ++i) b2 += source[i] * source[i];
    if (b2 > 0) rel2 = op.precision / b2;
  }
  p.tol = std::sqrt(rel2);
  p.max_iter = op.max_iter;
  cvcb_solver_stats st;
  double *x[1] = {propagator};
  const double *b[1] = {source};
  const int rc = cvcb_solve(g.lat, x, b, 1, &p, &st);
  if (rc != CVCB_OK) {
    std::fprintf(stderr, "[tmLQCD_invert] op %d: %s (status %d, residual %.3e)\n", op_id,
                 cvcb_last_error(), rc, st.max_true_res);
    return 5;
  }
  const size_t n = (size_t)24 * g.T * g.LX * g.LY * g.LZ;
  const double scale = 1.0 / (2.0 * op.kappa);
  for (size_t i = 0; i < n; ++i) propagator[i] *= scale;
  if (g.verbose)
    std::printf("# [tmLQCD_invert] op %d: %d iterations, |b - Q x|/|b| = %.3e\n", op_id,
                st.iterations, st.max_true_res);
  if (write_prop) {
    char name[1024];
    std::snprintf(name, sizeof name, "%s.%.4d.%.2d.inverted", g.prop_prefix.c_str(), g.nstore,
                  g.nwritten++);
    if (cvcb_write_propagator(propagator, name, 64, g.T, g.LX, g.LY, g.LZ, nullptr) != CVCB_OK)
      return 6;
  }
  return 0;
}

int tmLQCD_finalise() {
  if (g.lat) cvcb_lattice_destroy(g.lat);
  g.lat = nullptr;
  g.gauge.clear();
  g.gauge.shrink_to_fit();
  g.init = false;
  return 0;
}

int tmLQCD_get_gauge_field_pointer(double **gf) {
  if (!g.init || !gf) return 1;
  *gf = g.gauge.data();
  return 0;
}

int tmLQCD_get_mpi_params(tmLQCD_mpi_params *params) {
  if (!g.init || !params) return 1;
  std::memset(params, 0, sizeof *params);
  params->nproc = params->nproc_t = params->nproc_x = params->nproc_y = params->nproc_z = 1;
  params->omp_num_threads = 1;
  return 0;
}

int tmLQCD_get_lat_params(tmLQCD_lat_params *params) {
  if (!g.init || !params) return 1;
  params->LX = g.LX;
  params->LY = g.LY;
  params->LZ = g.LZ;
  params->T = g.T;
  params->nstore = g.nstore;
  params->nsave = g.nsave;
  params->no_operators = (unsigned)g.ops.size();
  return 0;
}

}  // extern "C"
