// Coefficient plan of the contraction's Z columns (contract.cu), shared with
// the adjoint (adjoint.cu).
#pragma once

#include "cvcb_internal.h"

namespace cvcb {

struct ZTerm {
  int src;       // column of the dn block (0..59 within fields[60..119])
  double2 coef;  // conj(k us)
};
struct ZPlan {
  ZTerm t[24][6];  // 24 columns (2 parts x 12), 6 terms each
};

// Host-side description of each plan term (for the source-link gradient):
// the term's coefficient is conj(k * us), us = Usource[nu](ia,ib) (part 0)
// or conj(Usource[nu](ib,ia)) (part 1).
struct ZMeta {
  double2 k;
  int ia, ib, part;
};

// plans[nu], Us[nu] (phased source links); meta (may be null) receives
// 4 x 24 x 6 entries indexed ((nu * 24 + col) * 6 + term).
int make_zplans(cvcb_lattice *L, int src, ZPlan plans[4], double Us[4][18], ZMeta *meta);
int launch_cvc_z(cvcb_lattice *L, double2 *Z, const double2 *dn, const ZPlan &plan);

}  // namespace cvcb
