/*
 * cm3d_oracle.h -- CPU restatement of CM3D's nonbonded force path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the GPU engine is compared
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it; the product never does.
 *
 * Each routine restates one CM3D routine (cited in cm3d_oracle.c) on the
 * arrays of a cm3d_nb_system, in CM3D's own operation order: the lists are
 * built in the link-cell traversal order of get_ngbr/get_ngbr_e, the pair
 * kernels work through the lists in chunks of nlen pairs exactly as
 * force_ter/force_ter_e hand them to force_npol/force_e, and the Ewald sum
 * uses fk_ewald's kc-recursion.  Compiled with -ffp-contract=off it
 * reproduces the reference's forces, energies and virials bit for bit.
 */
#ifndef CM3D_ORACLE_H
#define CM3D_ORACLE_H

#include "../include/cm3d_nb.h"

typedef struct orc orc;

/* ncells: NGBR.ncells (keyword ncell_div, odd); nocell_all: 1 = link cells
   (CM3D's default), 0 = all pairs; nlen: SIMPARMS.nlen (chunk length) */
orc *orc_create(const cm3d_nb_system *sys, int ncells, int nocell_all, int nlen);
void orc_destroy(orc *o);

void orc_set_positions(orc *o, const double *px, const double *py, const double *pz);
void orc_get_positions(orc *o, double *px, double *py, double *pz);
void orc_set_velocities(orc *o, const double *vx, const double *vy, const double *vz);
void orc_get_velocities(orc *o, double *vx, double *vy, double *vz);
/* which: 0 fxl, 1 fxs, 2 fxa (as stored: accelerations after rmass) */
void orc_get_forces(orc *o, int which, double *fx, double *fy, double *fz);
void orc_zero_forces(orc *o, int which);

void orc_get_ngbr(orc *o);
long long orc_list_count(orc *o, int which);
void orc_get_list(orc *o, int which, int *ip, int *jp);

void orc_force(orc *o, int iflg);
void orc_force_ter(orc *o, int iflg);
void orc_force_ter_e(orc *o, int iflg);
void orc_fk_ewald(orc *o);
void orc_ecorr(orc *o);
void orc_fbond(orc *o);
void orc_fbend(orc *o);
void orc_fbondx(orc *o);
void orc_ftors(orc *o);
void orc_fonfo(orc *o);
void orc_rmass(orc *o, int which);

/* out[0..]: see orc_get_energies in cm3d_oracle.c (same layout as
   cm3d_nb_energies) */
void orc_get_energies(orc *o, cm3d_nb_energies *e);
void orc_step_init(orc *o);
void orc_step(orc *o, int istep0, int nsteps);
/* the Nose-Hoover chain state (ntherm x nchain each) */
void orc_get_nhc(orc *o, double *eta, double *veta);
long long orc_rebuilds(orc *o);
long long orc_resets(orc *o);
long long orc_underflows(orc *o);

#endif
