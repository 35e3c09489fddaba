/* Input-file reader for the oracle build of the reference contraction program.
 *
 * Test infrastructure only.  The reference's flex parser cannot be built here
 * (no lex, and the pre-generated read_input_parser_cvc.c is empty in the
 * mounted tree), so this file supplies read_input_parser() with the same
 * contract as read_input_parser_cvc.l:979-1001: set the defaults via
 * set_default_input_values() (cvc_utils.c:1706), then read `key = value`
 * lines.  Only the keys the contraction program needs are understood; each
 * assigns the same global as the corresponding flex rule
 * (read_input_parser_cvc.l:317-470).  Unknown keys are ignored.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "global.h"
#include "cvc_utils.h"
#include "read_input_parser.h"

namespace cvc {

int verbose = 0;
int myverbose = 0;
double ft_rmax[4];

static void trim(char *s) {
  char *p = s;
  while (*p == ' ' || *p == '\t') p++;
  memmove(s, p, strlen(p) + 1);
  size_t n = strlen(s);
  while (n > 0 && (s[n - 1] == ' ' || s[n - 1] == '\t' || s[n - 1] == '\n' || s[n - 1] == '\r'))
    s[--n] = '\0';
}

static void apply(const char *k, const char *v) {
  if (!strcmp(k, "T")) T_global = atoi(v);
  else if (!strcmp(k, "L")) L = atoi(v);
  else if (!strcmp(k, "LX")) LX = atoi(v);
  else if (!strcmp(k, "LY")) LY = atoi(v);
  else if (!strcmp(k, "LZ")) LZ = atoi(v);
  else if (!strcmp(k, "kappa")) g_kappa = atof(v);
  else if (!strcmp(k, "mu")) g_mu = atof(v);
  else if (!strcmp(k, "Nconf")) Nconf = atoi(v);
  else if (!strcmp(k, "BCangleT")) BCangle[0] = atof(v);
  else if (!strcmp(k, "BCangleX")) BCangle[1] = atof(v);
  else if (!strcmp(k, "BCangleY")) BCangle[2] = atof(v);
  else if (!strcmp(k, "BCangleZ")) BCangle[3] = atof(v);
  else if (!strcmp(k, "filename_prefix")) strcpy(filename_prefix, v);
  else if (!strcmp(k, "filename_prefix2")) strcpy(filename_prefix2, v);
  else if (!strcmp(k, "filename_prefix3")) strcpy(filename_prefix3, v);
  else if (!strcmp(k, "gaugefilename_prefix")) strcpy(gaugefilename_prefix, v);
  else if (!strcmp(k, "outfile_prefix")) strcpy(g_outfile_prefix, v);
  else if (!strcmp(k, "source_location")) g_source_location = atoi(v);
  else if (!strcmp(k, "format")) format = atoi(v);
  else if (!strcmp(k, "solver_precision")) solver_precision = atof(v);
  else if (!strcmp(k, "niter_max")) niter_max = atoi(v);
  else if (!strcmp(k, "propagator_position")) g_propagator_position = atoi(v);
}

int read_input_parser(char *conf_file) {
  set_default_input_values();
  FILE *f = fopen(conf_file, "rt");
  if (!f) return 2;
  char line[512];
  while (fgets(line, sizeof line, f)) {
    char *eq = strchr(line, '=');
    if (!eq || line[0] == '#') continue;
    *eq = '\0';
    char key[256], val[256];
    strncpy(key, line, 255); key[255] = '\0';
    strncpy(val, eq + 1, 255); val[255] = '\0';
    trim(key); trim(val);
    apply(key, val);
  }
  fclose(f);
  return 0;
}

int reread_input_parser(char *conf_file) {
  FILE *f = fopen(conf_file, "rt");
  if (!f) return 2;
  fclose(f);
  return read_input_parser(conf_file);
}

}  // namespace cvc
