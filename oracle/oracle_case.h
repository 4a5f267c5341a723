/* Case description shared by the CPU oracle (oracle/lbm_oracle.c) and the
 * reference build (oracle/ref_driver.cpp).  TEST INFRASTRUCTURE ONLY: the
 * product library never includes this header.
 *
 * Field names follow the reference's input keys:
 *   lattice  : lbm2d|lbm3d.{ndir,wis,wim,dirx,diry,dirz}
 *              (Source/Core/AmrCoreLBM.cpp:1212-1236, w = wis/wim)
 *   geometry : amr.n_cell, geometry.prob_lo/prob_hi/is_periodic
 *   BCs      : amrbc.bc_lo/bc_hi + bc_{lo,hi}_<d>_{rho,ux,uy,uz}_val
 *              (Source/Core/AmrCoreLBM.cpp:254-330)
 *   physics  : lbmPhysicalParameters.nu, lbm.prescribed_force
 *              (Source/Core/AmrCoreLBM.cpp:1238-1265)
 *   IB       : ibm.* / MarkerIBParams (Source/IBM/MarkerIBParams.H:8-132)
 */
#ifndef ILBM_ORACLE_CASE_H
#define ILBM_ORACLE_CASE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ILBM_MAX_Q 27

typedef struct {
  int dim; /* 2 or 3 */
  int q;
  double cx[ILBM_MAX_Q], cy[ILBM_MAX_Q], cz[ILBM_MAX_Q];
  double wis[ILBM_MAX_Q], wim[ILBM_MAX_Q];
  int n_cell[3];
  double prob_lo[3], prob_hi[3];
  int periodic[3];
  int bc_lo[3], bc_hi[3]; /* AMReX BCType codes: 0 int_dir, 2 foextrap, 3 ext_dir, 1001 user_1, 1002 user_2 */
  double bc_lo_rho[3], bc_lo_ux[3], bc_lo_uy[3], bc_lo_uz[3];
  double bc_hi_rho[3], bc_hi_ux[3], bc_hi_uy[3], bc_hi_uz[3];
  double nu;
  int use_prescribed_force;
  double prescribed_force[3];
  int nghost; /* ghost width of the population/macro MultiFabs (3 in the reference) */
} ilbm_case;

typedef struct {
  /* MarkerIBParams (Source/IBM/MarkerIBParams.H) */
  int coupling_method; /* 0 explicit, 1 ivc, 2 explicit_diag */
  int delta_type;      /* 0/4 = 4-point, 1/3 = 3-point */
  int loop_ns;
  double mdf_relax;
  double explicit_diag_eps;
  int geometry_type; /* 0 cylinder/sphere, 1 box, 2 user_defined (pitching NACA) */
  double box_xlo, box_xhi, box_ylo, box_yhi, box_zlo, box_zhi, box_ds;
  int box_lid_only;
  double box_lid_ux, box_lid_uy, box_lid_uz, box_wall_tol;
  int n_marker;
  double rd;
  double ubx, uby, ubz, omx, omy, omz;
  double ivc_diag_reg;
  int ivc_rebuild_matrix;
  int renormalize_delta;
  /* body (ibm.x0, y0, z0, R) */
  double x0, y0, z0, R;
  /* force evaluation (ibm.force_eval_method: 0 momentum_exchange, 1 eulerian, 2 marker) */
  int force_eval_method;
  double U0; /* lbmPhysicalParameters.U0 */
} ilbm_ib_case;

/* One ComputeIBForce record (Source/Core/AmrCoreLBM.cpp:456-631):
 * [Fx_tc, Fy_tc, Fz_tc, Cd, Cl, Cz,
 *  Fx_raw, Fy_raw, Fz_raw, Fx_eul, Fy_eul, Fz_eul,
 *  Fx_marker, Fy_marker, Fz_marker, Fx_me, Fy_me, Fz_me] */
#define ILBM_FORCE_REC 18

#ifdef __cplusplus
}
#endif
#endif
