/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it, and only as the checker. The product never links it.
 *
 * A plain-C restatement of the reference's CPU path for the per-timestep hot path of cellGPU
 * (abaso/cellGPU), FP64 throughout, each function citing the reference file:line it follows.
 * Layout conventions are the reference's: neighbour rows n_idx(k,c) = c*K + k
 * (inc/utility/indexer.h:38-41), positions as interleaved (x,y) doubles.
 */
#ifndef CG_ORACLE_H
#define CG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- periodic square box, reference semantics (inc/utility/gpubox.h:131-179) ---- */
void cgo_min_dist(const double *box, const double *p1, const double *p2, double *out);
void cgo_put_in_box(const double *box, double *p);

/* ---- Delaunay (CGAL boundary, inc/models/DelaunayCGAL.h; src/models/DelaunayCGAL.cpp:8-48,164-229) ----
 * Star of the origin among m relative points (rel[2*i], rel[2*i+1]); writes candidate indices of the
 * Delaunay neighbours in counter-clockwise order to out (capacity cap); returns the count, or -1 if the
 * origin is not enclosed, or -2 on overflow. Gift-wrapping with exact predicates. */
int cgo_local_star(int m, const double *rel, int cap, int *out);
/* Brute-force variant (O(m^3) empty-circle enumeration), used to cross-check cgo_local_star. */
int cgo_local_star_bruteforce(int m, const double *rel, int cap, int *out);
/* Full periodic Delaunay triangulation of N points in a square box of side L. Rows are CCW and
 * rotated to start at the smallest neighbour index. Returns 0, or <0 on failure (K too small: -2). */
int cgo_periodic_delaunay(int N, const double *pos, const double *box, int K, int *nn, int *nbr);
/* Count of cells whose stored row differs from the exact Delaunay star (canonical rotation). */
int cgo_topology_mismatch(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr);

/* ---- Voronoi model (src/models/voronoiModelBase.cpp:783-846; src/models/voronoiQuadraticEnergy.cpp:172-397) ---- */
void cgo_voronoi_geometry(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                          double *AP);
int cgo_voronoi_forces(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                       const double *AP, const double *APpref, double KA, double KP, double *F);
double cgo_voronoi_energy(int N, const double *AP, const double *APpref, double KA, double KP);
int cgo_voronoi_tension_forces(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                               const double *AP, const double *APpref, double KA, double KP, const int *ctype,
                               int ntypes, double gamma, const double *tmat, double *F);
double cgo_voronoi_tension_energy(int N, const double *pos, const double *box, int K, const int *nn,
                                  const int *nbr, const double *AP, const double *APpref, double KA, double KP,
                                  const int *ctype, int ntypes, double gamma, const double *tmat);

/* ---- self-propelled particle dynamics, CPU semantics (src/updaters/selfPropelledParticleDynamics.cpp:67-101) ---- */
void cgo_spp_step(int N, double *pos, const double *box, const double *F, double *theta, const double *motility,
                  const double *noise, double dt, double mu);
/* Full SPP timestep of the Voronoi model with supplied noise: forces on the current topology, integrate,
 * move, retriangulate (Delaunay is unique, so local repair and global retriangulation agree).
 * noise has n_steps*N normals. Returns 0 or <0 on a triangulation failure. */
int cgo_voronoi_spp_run(int N, double *pos, const double *box, int K, int *nn, int *nbr, double *theta,
                        const double *motility, const double *APpref, double KA, double KP, double dt,
                        double mu, int n_steps, const double *noise, double *F_out, double *AP_out);

/* ---- Brownian dynamics (src/updaters/brownianParticleDynamics.cpp:92-109) ---- */
void cgo_brownian_disp(int N, const double *F, const double *noise2, double dt, double mu, double T,
                       double *disp);

/* ---- vertex model ---- */
/* Vertex topology from the Delaunay dual (src/models/vertexModelBase.cpp:115-229): vertices are the
 * circumcentres of the Delaunay triangles. Returns Nv (=2N) or <0. Triangles are enumerated with
 * the smallest cell index first (canonical order); cv rows are CCW starting from the vertex of the
 * triangle (c, nbr[0], nbr[1]). */
int cgo_vertex_from_delaunay(int N, const double *pos, const double *box, int K, const int *nn, const int *nbr,
                             int vmax, double *vpos, int *vn, int *vcn, int *cvn, int *cv);
/* geometry (src/models/vertexModelBase.cpp:248-297), forces (src/models/vertexQuadraticEnergy.cpp:71-113,
 * inc/utility/functions.h:330-354) */
void cgo_vertex_geometry(int Nc, const double *vpos, const double *box, int vmax, const int *cvn, const int *cv,
                         double *AP);
void cgo_vertex_forces(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                       const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                       double KP, double *F);
void cgo_vertex_tension_forces(int Nc, int Nv, const double *vpos, const double *box, int vmax, const int *cvn,
                               const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                               double KP, const int *ctype, int ntypes, double gamma, const double *tmat,
                               double *F);
double cgo_vertex_tension_energy(int Nc, const double *vpos, const double *box, int vmax, const int *cvn,
                                 const int *cv, const int *vcn, const double *AP, const double *APpref, double KA,
                                 double KP, const int *ctype, int ntypes, double gamma, const double *tmat);
/* Sequential T1 sweep (src/models/vertexModelBase.cpp:507-787). Returns the number of flips performed,
 * writes each flip's (vertex1, vertex2) to events (capacity max_events pairs). Returns -2 if a cell
 * would exceed vmax vertices. */
int cgo_vertex_t1(int Nc, int Nv, double *vpos, const double *box, double threshold, int vmax, int *vn,
                  int *vcn, int *cvn, int *cv, int max_events, int *events);
/* Brownian step of the vertex model with supplied noise (2 normals per vertex per step, x then y) */
int cgo_vertex_brownian_run(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn,
                            int *cvn, int *cv, const double *APpref, double KA, double KP, double dt,
                            double mu, double T, double t1_threshold, int n_steps, const double *noise,
                            double *F_out, double *AP_out, int *n_t1_out);

/* self-propelled vertex model with supplied noise (one normal per cell per step) */
int cgo_vertex_spp_run(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn,
                       int *cvn, int *cv, const double *APpref, double KA, double KP, double *theta,
                       const double *motility, double dt, double mu, double t1_threshold, int n_steps,
                       const double *noise);

/* ---- FIRE (src/updaters/EnergyMinimizerFIRE2D.cpp:120-151,212-284), CPU conventions ---- */
typedef struct {
    double dt, dt_max, dt_min, dt_inc, dt_dec, alpha, alpha_start, alpha_dec, force_cutoff;
    int n_min, max_iterations;
    /* outputs / state */
    int iterations, n_since_negative_power;
    double power, force_max;
} cgo_fire_params;
/* model: 0 = Voronoi (dofs = cells), 1 = vertex (dofs = vertices). For the vertex model the
 * topology arrays are vn,vcn,cvn,cv and t1_threshold applies; for Voronoi nn/nbr with capacity K. */
int cgo_fire_voronoi(int N, double *pos, const double *box, int K, int *nn, int *nbr, const double *APpref,
                     double KA, double KP, cgo_fire_params *prm, double *vel, double *F_out,
                     double *AP_out);
int cgo_fire_vertex(int Nc, int Nv, double *vpos, const double *box, int vmax, int *vn, int *vcn, int *cvn,
                    int *cv, const double *APpref, double KA, double KP, double t1_threshold,
                    cgo_fire_params *prm, double *vel, double *F_out, double *AP_out);

#ifdef __cplusplus
}
#endif
#endif
