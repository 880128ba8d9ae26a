// Device-side views of the molecule-type tables and of a batch of independent
// systems.  Shared by the kernels (pbsam_kernels.cu) and the C-ABI host code
// (pbsam_api.cu).
#pragma once
#include "pbsam_device.cuh"

namespace pbsam {

// Solver parameters: the reference's compile-time tolerances and cutoffs made
// runtime values (src/molecule.cpp:6-13, src/expcenter.cpp:16-22,
// src/BDnam.cpp:82,138-139, src/molecule.h:22).
struct SolveParams {
  double max_polar_dev;    // outer stop: avg dev > max_polar_dev^2 continues
  double solve_tol;        // inner F/H fixed-point stop
  int solve_max_ct;        // inner iteration cap
  int max_pol_rounds;      // outer sweep cap
  double inter_cut;        // inter-molecular polarization cutoff (surface gap)
  double interact_cut;     // inter-molecular interaction cutoff
  double min_sep_numeric;  // intra pairs closer than this re-expand numerically
  double idiel, sdiel;
  int exact;               // 1: exact form (direct inner solves, full sweeps, adjoint forces)
  double exact_tol;        // exact form: sweep stop (root-mean-square relative change)
  double exact_relax;      // exact form: over-relaxation factor of the sweeps' updates
  double box;              // > 0: edge of a cubic periodic box (minimum-image displacements)
};

// minimum image of a displacement in a cubic periodic box of edge box
// (CSystem::pbcPos, src/system.cpp:46-55); box <= 0: no periodic box
__device__ __forceinline__ void min_image(double box, double *d)
{
  if (box > 0.0)
    for (int k = 0; k < 3; k++) d[k] = d[k] - box * round(d[k] / box);
}

// Per-sphere constant block layout inside TypeView::cst (NP doubles each).
enum { CST_H1 = 0, CST_F1, CST_H2, CST_F2, CST_LH1, CST_LF1, CST_LH2, CST_LF2, CST_INVH, CST_CHGH, CST_N };

// Molecule types, concatenated over all types ("type sphere" index ts).
struct TypeView {
  int ntypes, TS;
  const int *type_off;     // [ntypes+1] first type sphere of each type
  const double *maxR;      // [ntypes]
  const double *cen;       // [TS][3] sphere centre in the molecule frame
  const double *rad;       // [TS]
  const int *spx_off;      // [TS+1] exposed surface points (CSR)
  const double *spx;       // [TP][3] relative to the sphere centre
  const int *nspx;         // [TS] number of generated points (quadrature weight 4pi/nspx)
  const double *Fself, *Hself;       // [TS][NP2]
  const double *hself_scale;         // [TS]  scale value read with Hself
  double *qFself, *qHself;           // [TP]
  double *tFself, *tHself;           // [TS]
  double *LFintra, *LHintra, *LFfar, *LHfar;   // [TS][NP2]
  const int *near_off, *near;        // CSR: intra near list (type sphere indices within the type)
  double *Dfix, *Vfix;               // [TS][NP2]
  double *cst;                       // [TS][CST_N][NP]
  const double *imat;                // [TS][NP2][ld] row-major (see imat_stride)
  // charges of each type (for the fixed-charge expansions)
  const int *chg_off;      // [ntypes+1]
  const double *chg_pos;   // [TQ][3] relative to the molecule centre
  const double *chg;       // [TQ]
  const int *chg_lab;      // [TQ] sphere (within the type) each charge is assigned to
  double *Eass;            // [TS][NP2] multipole of the assigned charges (self-polarization start)
  // coefficient tables of the intra pairs: one entry per ordered pair (ki, kj != ki)
  // of each type, entry pair_off[ts] + (kj < ki ? kj : kj - 1)
  const int *pair_off;     // [TS+1]
  double2 *pR;             // [TE][rot_off(NP)]
  double *pTH, *pTF;       // [TE][tr_off(NP)] screened / unscreened translation
  double *pS;              // [TE][16] rotation scalars
  const double *Gdir;      // [TS][2NP2][2NP2] row-major or null: the inner fixed point solved for
                           // (fb, hb) -> (F, H) (exact form, pbsam_direct_kernel)
  const int *nslot;        // [near entries] operator slot of each intra near entry, -1 if none
  const int *nkind;        // [slots] 0: analytic pair (rotation + translation), 1: numeric
  const double *Nmat;      // [slots][2][NP2][NP2] row-major or null: the near-field operators
                           // N_F, N_H of the intra near pairs (exact form, pbsam_nummat_kernel)
  const double *spang;     // [TP][4] or null: cos t, sin t, cos phi, sin phi of every exposed
                           // point (exact form, pbsam_spang_kernel)
};

// Batch of B independent systems with the same list of molecules.
struct BatchView {
  int B, nmol, S, SP;        // systems, molecules, spheres and points per system
  const int *mol_type;       // [nmol]
  const int *mol_off;        // [nmol+1]
  const int *sph_ts;         // [S]
  const int *sph_mol;        // [S]
  const int *pt_off;         // [S+1]
  const double *pos, *quat;  // [B][nmol][3], [B][nmol][4]
  double *F, *H, *Hrot, *HselfRot, *LS, *LFS, *LHS;   // [B][S][NP2]
  double *hscale, *tF, *tH, *maxgF, *maxgH, *dev;     // [B][S]
  double *qF, *qH;           // [B][SP]
  double *gFp, *gHp;         // [B][SP][3]
  double *gLHN, *gH;         // [B][S][3][NP2]
  double *cenRot;            // [B][S][3]
  double *Hlab;              // [B][S][NP2] H rotated to the lab frame (lab-frame energy)
  int *ipol, *ipol_n, *iact, *iact_n;        // [B][S][S], [B][S]
  int *interMol, *interMol_n;                // [B][nmol][S], [B][nmol]
  int *intraPol, *intraPol_n, *intraAct, *intraAct_n;
  int *interX;               // [B][nmol]
  double *gFw, *gHw, *gHrotw, *tGw;          // [B][S][3][NP2] gradient work set
  int *gkey;                 // [B][S]
  double *dgrad;             // [B][S]
  double2 *molR;             // [B][nmol][rot entries at NP]
  double *molRS;             // [B][nmol][8] rotation state scalars
  double *sep;               // [B][S][S] sphere-sphere surface gaps
  double *scr;               // [B][crew][scr_stride]: one scratch block per CTA
  long long scr_stride;
  int *dorder;               // [B][crew][S] pair orders of a CTA's share of a gradient list
  double *wscr;              // [B][crew][16 warps][wscr_stride]: per-warp scratch of the
  long long wscr_stride;     // gradient re-expansion lists (pairs of low order)
  int crew;                  // CTAs per system
  double *force, *torque, *energy;  // [B][nmol][3], [B][nmol][3], [B]
  double *dpos, *drot;       // [B][nmol][3]: dU/dpos, dU/domega (lab frame) of the last backward pass
  int *status;               // [B]
  const int *fmask;          // [B] or null: systems with fmask[b] == 0 are skipped by the
                             // force kernel (Brownian dynamics steps without forces)
  int *stats;                // [B][8]: sweeps, inner iterations, solves, grad solves, ...
  double *tphase;            // [B][8] device time per phase (ns): solve, surface charges,
                             // numeric near field, analytic intra, inter LS, gradient DTA,
                             // gradient-solve re-expansions, total
};

enum {
  PBSAM_STATUS_OK = 0,
  PBSAM_STATUS_OVERLAP = 1,
  PBSAM_STATUS_NOT_CONVERGED = 2,
  PBSAM_STATUS_NAN = 3,
};

struct Ctx {
  Tab T;
  TypeView tv;
  BatchView bv;
  SolveParams prm;
  int do_energy;
};

}  // namespace pbsam
