/*
 * sod2d_host.h -- host-side set-up for the SOD2D spectral-element hot path.
 *
 * These routines restate, in C, the set-up work the SOD2D Fortran solver does
 * before its time loop (shape functions, Jacobians, lumped mass, element
 * sizes) and add a synthetic periodic-cube mesh generator that stands in for
 * the gmsh -> HDF5 mesh pipeline (tool_meshConversorPar), which needs HDF5.
 *
 * Every array uses the reference's Fortran layout: column-major, and element
 * connectivity holds 1-based node ids.  Sizes below: P = element order,
 * n = (P+1)^3 nodes (= Gauss points) per element, E elements, N nodes.
 *
 * All functions return 0 on success and a negative code on a bad argument.
 * Nothing here needs a GPU.
 */
#ifndef SOD2D_HOST_H
#define SOD2D_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss-Lobatto-Legendre nodes (ascending, natural order) and weights in
 * FP64.  Replaces ZELEGL/WELEGL, src/lib_sod2d/sources/mod_maths.f90:41-106. */
int sod_host_gll(int porder, double *xi, double *w);

/* Element-local node numbering.  atoIJK(c) gives the element-local node
 * number of tensor position c, c running k-outer, i-middle, j-inner over the
 * SOD2D 1-D order [-1, +1, interior...] (the meaning of mesh_a2ijk used at
 * CFDSolverBase.f90:1531).  kind 0: the 8 hex vertices first in gmsh vertex
 * order, then the remaining positions in c order.  kind 1: as kind 0 with the
 * non-vertex numbers shuffled by a seeded permutation (exercises callers that
 * pass arbitrary orderings, e.g. gmsh's). */
int sod_host_atoijk(int porder, int kind, uint64_t seed, int *atoIJK);

/* invAtoIJK(P+1,P+1,P+1) and gmshAtoI/J/K(n) from atoIJK.  Replaces
 * atoIJKInverse, src/lib_sod2d/sources/mod_geom.f90:127-148. */
int sod_host_atoijk_inverse(int porder, const int *atoIJK, int *invAtoIJK,
                            int *gmshAtoI, int *gmshAtoJ, int *gmshAtoK);

/* Shape-function tables at the GLL Gauss points, computed in FP64 and rounded
 * to FP32 as CFDSolverBase_evalShapeFunctions does (CFDSolverBase.f90:1468-1619,
 * hex_highorder elem_hex.f90:22-43, TripleTensorProduct mod_maths.f90:325-373):
 *   xgp(n,3), wgp(n), Ngp(n,n), dNgp(3,n,n), dlxigp_ip(n,3,P+1).
 * Any output pointer may be NULL. */
int sod_host_shape_tables(int porder, const int *atoIJK, float *xgp, float *wgp,
                          float *Ngp, float *dNgp, float *dlxigp_ip);

/* Sizes of the periodic cube mesh of nx*ny*nz hexahedra of order P:
 * npoin counts the periodic duplicate (slave) nodes, npoin_w only masters. */
int sod_host_cube_sizes(int porder, int nx, int ny, int nz, int *nelem,
                        int *npoin, int *npoin_w);

/* Periodic cube [0,L]^3 of nx*ny*nz hexahedra with GLL nodes.  Outputs, in
 * the layout of the reference mesh arrays (mod_mpi_mesh.f90):
 *   coord(N,3) FP32, connecOrig(E,n) (true nodes, for Jacobians),
 *   connecWork(E,n) (slave ids replaced by their master, as
 *   create_working_lists_parallel does, mod_meshConversorTool.f90:4917-5008),
 *   lpoin_w(N_w) (1-based master ids, ascending).
 * jitter > 0 moves every element-interior node by a seeded uniform offset of
 * +-jitter times the local GLL spacing in each direction (the mesh stays
 * conforming and periodic).  elem_shuffle != 0 permutes the element order. */
int sod_host_cube_mesh(int porder, int nx, int ny, int nz, double L,
                       double jitter, uint64_t seed, int elem_shuffle,
                       const int *atoIJK, float *coord, int *connecOrig,
                       int *connecWork, int *lpoin_w);

/* He(3,3,n,E) = J^-1 and gpvol(1,n,E) = w*det(J).  Replaces elem_jacobian,
 * src/lib_sod2d/sources/jacobian_oper.f90:7-139 (FP64 Jacobian from FP32
 * products, cofactor inverse, rounded to FP32). */
int sod_host_elem_jacobian(int porder, int nelem, int npoin,
                           const int *connecOrig, const float *coord,
                           const float *dNgp, const float *wgp, float *gpvol,
                           float *He);

/* Lumped mass Ml(N) = sum of gpvol over connecWork, invMl = 1/Ml on working
 * nodes (0 elsewhere).  Replaces lumped_mass_spectral (mass_matrix.f90:11-42)
 * and CFDSolverBase.f90:1773-1781.  Also returns the FP64 domain volume. */
int sod_host_lumped_mass(int porder, int nelem, int npoin, int npoin_w,
                         const int *connecWork, const int *lpoin_w,
                         const float *gpvol, float *Ml, float *invMl,
                         double *vol_total);

/* helem(E): smallest vertex-to-vertex edge length (char_length,
 * mod_geom.f90:13-37); helem_l(E,n): distance from each node to the nearest
 * other node of its element (char_length_spectral, mod_geom.f90:39-66).
 * Both read connecOrig (first 8 local nodes must be the vertices). */
int sod_host_char_length(int porder, int nelem, int npoin,
                         const int *connecOrig, const float *coord,
                         float *helem, float *helem_l);

/* lelpn(N): number of elements sharing each node through connecWork
 * (elemPerNode, mod_geom.f90:87-117). */
int sod_host_elem_per_node(int porder, int nelem, int npoin,
                           const int *connecWork, int *lelpn);

/* Compressible Taylor-Green vortex initial state in FP32, as
 * TGVCompSolver_evalInitialConditions (TGVCompSolver.f90:154-214) with the
 * derived constants of TGVCompSolver_initializeParameters (:128-146).
 * Outputs per node (level 2 of the reference's 4-level arrays): rho, u(N,3),
 * q(N,3), pr, E, Tem, e_int, csound, machno (|u|^2/c, as the reference), eta.
 * consts[0..7] receives Rgas, Cp, rho0, P0, mu_factor, gamma, Prt, Ma. */
int sod_host_tgv_comp_init(int npoin, const float *coord, float Ma, float V0,
                           float L, float T0, float Re, float gamma_gas,
                           float Prt, float *rho, float *u, float *q,
                           float *pr, float *E, float *Tem, float *e_int,
                           float *csound, float *machno, float *eta,
                           float *consts);

#ifdef __cplusplus
}
#endif
#endif
