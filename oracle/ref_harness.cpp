// TEST INFRASTRUCTURE ONLY -- a C front end to the reference's own CPU path, compiled from the
// reference sources in place (oracle/Makefile.ref) with the DelaunayCGAL stand-in of oracle/shim.
// Used to pin the C oracle against the reference's code and, in bench.py's reference arm, as the
// CPU baseline. Nothing here is shipped.
//
// Noise: the reference's CPU updaters draw N(0,1) deviates from their own noiseSource, which with
// setReproducible(true) is a std::mt19937 seeded 13377 with a fresh std::normal_distribution per
// draw (inc/utility/noiseSource.h:22-33, src/utility/noiseSource.cpp:29-38). ref_reproducible_normals
// replays that stream (same standard-library generator and distribution) so the GPU can be fed the
// identical deviates.
#include <memory>
#include <random>
#include <vector>

#include "EnergyMinimizerFIRE2D.h"
#include "Simulation.h"
#include "brownianParticleDynamics.h"
#include "dynamicalFeatures.h"
#include "selfPropelledParticleDynamics.h"
#include "vertexQuadraticEnergy.h"
#include "voronoiQuadraticEnergy.h"
#include "voronoiQuadraticEnergyWithTension.h"
#include "vertexQuadraticEnergyWithTension.h"

namespace {

// exposes the protected retriangulation entry points of voronoiModelBase
class RefVoronoi : public VoronoiQuadraticEnergy {
  public:
    RefVoronoi(int n, Dscalar A0, Dscalar P0) : VoronoiQuadraticEnergy(n, A0, P0, true) {}
    int neigh_max() const { return neighMax; }
    void retriangulate()
    {
        globalTriangulationCGAL();
        resetLists();
        allDelSets();
    }
};

// the line-tension model, with the same retriangulation access
class RefVoronoiTension : public VoronoiQuadraticEnergyWithTension {
  public:
    RefVoronoiTension(int n, Dscalar A0, Dscalar P0) : VoronoiQuadraticEnergyWithTension(n, A0, P0, true) {}
    void retriangulate()
    {
        globalTriangulationCGAL();
        resetLists();
        allDelSets();
    }
};

// exposes the protected vertex-model arrays
// (the tension subclass computes the plain forces while its tension is off, so one class serves
// both uses)
class RefVertex : public VertexQuadraticEnergyWithTension {
  public:
    RefVertex(int n, Dscalar A0, Dscalar P0) : VertexQuadraticEnergyWithTension(n, A0, P0, true, false) {}
    void dirty() { forcesUpToDate = false; }
    int cells() const { return Ncells; }
    int vmax() const { return vertexMax; }
    GPUArray<int> &cell_vertices() { return cellVertices; }
};

struct RefSystem {
    std::shared_ptr<RefVoronoi> voro;
    std::shared_ptr<RefVertex> vertex;
    std::shared_ptr<Simulation> sim;
    std::shared_ptr<simpleEquationOfMotion> eom;
    std::shared_ptr<EnergyMinimizerFIRE> fire;
};

template <typename T>
void to_host(GPUArray<T> &a, T *out, int n)
{
    ArrayHandle<T> h(a, access_location::host, access_mode::read);
    for (int i = 0; i < n; ++i) out[i] = h.data[i];
}

}  // namespace

extern "C" {

// the deviates a reproducible noiseSource hands out, in order
void ref_reproducible_normals(int n, double *out)
{
    std::mt19937 gen(13377);
    for (int i = 0; i < n; ++i) {
        std::normal_distribution<> normal(0.0, 1.0);
        out[i] = normal(gen);
    }
}

// ---- Voronoi model ----------------------------------------------------------------------
void *ref_voronoi_new(int n, double A0, double P0)
{
    RefSystem *s = new RefSystem();
    s->voro = std::make_shared<RefVoronoi>(n, A0, P0);
    s->voro->setCPU(true);
    return s;
}

void ref_free(void *h) { delete reinterpret_cast<RefSystem *>(h); }

// positions (x,y pairs) and directors; retriangulates globally (CPU, stand-in CGAL boundary)
int ref_voronoi_set_state(void *h, const double *pos, const double *theta)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    std::vector<Dscalar2> p(n);
    for (int i = 0; i < n; ++i) p[i] = make_Dscalar2(pos[2 * i], pos[2 * i + 1]);
    s->voro->setCellPositions(p);
    if (theta) {
        ArrayHandle<Dscalar> hd(s->voro->cellDirectors, access_location::host, access_mode::overwrite);
        for (int i = 0; i < n; ++i) hd.data[i] = theta[i];
    }
    s->voro->retriangulate();
    return 0;
}

void ref_voronoi_set_motility(void *h, double v0, double Dr)
{
    reinterpret_cast<RefSystem *>(h)->voro->setv0Dr(v0, Dr);
}

void ref_voronoi_set_preferences(void *h, const double *pref)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    std::vector<Dscalar2> p(n);
    for (int i = 0; i < n; ++i) p[i] = make_Dscalar2(pref[2 * i], pref[2 * i + 1]);
    s->voro->setCellPreferences(p);
}

// forces, areas/perimeters and energy on the current topology
double ref_voronoi_forces(void *h, double *F, double *AP)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    s->voro->computeForces();
    to_host(s->voro->returnForces(), reinterpret_cast<Dscalar2 *>(F), n);
    to_host(s->voro->returnAreaPeri(), reinterpret_cast<Dscalar2 *>(AP), n);
    return s->voro->computeEnergy();
}

// particle exclusions (voronoiModelBase::setExclusions) and the external forces the force
// summation with exclusions stores for the excluded cells
void ref_voronoi_set_exclusions(void *h, const int *exes)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    std::vector<int> e(exes, exes + n);
    s->voro->setExclusions(e);
}

void ref_voronoi_external_forces(void *h, double *out)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    to_host(s->voro->external_forces, reinterpret_cast<Dscalar2 *>(out), n);
}

// the reference's observables on the current state: Simple2DCell::reportq, reportVarq and
// reportVarAP (after a force evaluation, which refreshes the areas and perimeters), and
// dynamicalFeatures::computeMSD / computeOverlapFunction of the current positions against `initial`
void ref_voronoi_observables(void *h, const double *initial, double cutoff, double *out)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    s->voro->computeForces();
    out[0] = s->voro->reportq();
    out[1] = s->voro->reportVarq();
    Dscalar2 v = s->voro->reportVarAP();
    out[2] = v.x;
    out[3] = v.y;
    GPUArray<Dscalar2> init((unsigned int)n, false);
    {
        ArrayHandle<Dscalar2> hi(init, access_location::host, access_mode::overwrite);
        for (int i = 0; i < n; ++i) hi.data[i] = make_Dscalar2(initial[2 * i], initial[2 * i + 1]);
    }
    dynamicalFeatures dyn(init, s->voro->Box);
    out[4] = dyn.computeMSD(s->voro->cellPositions);
    out[5] = dyn.computeOverlapFunction(s->voro->cellPositions, cutoff);
}

// state read-back: positions, directors, neighbour rows (K per row, -1 padded)
int ref_voronoi_get(void *h, double *pos, double *theta, int K, int *nn, int *nbr)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    to_host(s->voro->cellPositions, reinterpret_cast<Dscalar2 *>(pos), n);
    if (theta) to_host(s->voro->cellDirectors, theta, n);
    if (nn && nbr) {
        ArrayHandle<int> hn(s->voro->cellNeighborNum, access_location::host, access_mode::read);
        ArrayHandle<int> hb(s->voro->cellNeighbors, access_location::host, access_mode::read);
        int w = s->voro->neigh_max();
        for (int i = 0; i < n; ++i) {
            nn[i] = hn.data[i];
            for (int k = 0; k < K; ++k) nbr[(size_t)i * K + k] = (k < hn.data[i] && k < w) ? hb.data[i * w + k] : -1;
            if (hn.data[i] > K) return -2;
        }
    }
    return 0;
}

// SPP timesteps through Simulation::performTimestep, CPU branch, reproducible noise.
// local_repair: 1 = test-and-repair every step (setCPU(false)), 0 = global retriangulation every step
int ref_voronoi_spp_run(void *h, int steps, double dt, int local_repair)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->voro->getNumberOfDegreesOfFreedom();
    if (!s->sim) {
        auto spp = std::make_shared<selfPropelledParticleDynamics>(n);
        s->eom = spp;
        s->sim = std::make_shared<Simulation>();
        s->sim->setConfiguration(s->voro);
        s->sim->addUpdater(spp, s->voro);
        s->sim->setIntegrationTimestep(dt);
        s->sim->setCPUOperation(true);
        s->sim->setReproducible(true);
        if (local_repair) s->voro->setCPU(false);
    }
    for (int t = 0; t < steps; ++t) s->sim->performTimestep();
    return 0;
}

// ---- FIRE ---------------------------------------------------------------------------------
// one call of EnergyMinimizerFIRE::minimize (CPU branch) on the Voronoi or vertex system
int ref_fire(void *h, int vertex, double dt, double alpha_start, double dt_max, double dt_inc, double dt_dec,
             double alpha_dec, int n_min, double force_cutoff, int max_iterations)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    std::shared_ptr<Simple2DModel> m =
        vertex ? std::static_pointer_cast<Simple2DModel>(s->vertex) : std::static_pointer_cast<Simple2DModel>(s->voro);
    if (!s->fire) {
        s->fire = std::make_shared<EnergyMinimizerFIRE>(m);
        s->fire->setCPU();
    }
    s->fire->setDeltaT(dt);
    s->fire->setAlphaStart(alpha_start);
    s->fire->setDeltaTMax(dt_max);
    s->fire->setDeltaTInc(dt_inc);
    s->fire->setDeltaTDec(dt_dec);
    s->fire->setAlphaDec(alpha_dec);
    s->fire->setNMin(n_min);
    s->fire->setForceCutoff(force_cutoff);
    s->fire->setMaximumIterations(max_iterations);
    s->fire->minimize();
    return 0;
}

// ---- vertex model ---------------------------------------------------------------------------
// VertexQuadraticEnergy(n, A0, P0, reproducible) with the stand-in's periodic Delaunay dual
void *ref_vertex_new(int n, double A0, double P0)
{
    RefSystem *s = new RefSystem();
    s->vertex = std::make_shared<RefVertex>(n, A0, P0);
    s->vertex->setCPU();
    return s;
}

int ref_vertex_counts(void *h, int *nc, int *nv, int *vmax)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    *nc = s->vertex->cells();
    *nv = s->vertex->getNumberOfDegreesOfFreedom();
    *vmax = s->vertex->vmax();
    return 0;
}

int ref_vertex_get(void *h, double *cellpos, double *vpos, int *vn, int *vcn, int *cvn, int *cv)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int nc = s->vertex->cells(), nv = s->vertex->getNumberOfDegreesOfFreedom();
    if (cellpos) to_host(s->vertex->cellPositions, reinterpret_cast<Dscalar2 *>(cellpos), nc);
    to_host(s->vertex->vertexPositions, reinterpret_cast<Dscalar2 *>(vpos), nv);
    to_host(s->vertex->vertexNeighbors, vn, 3 * nv);
    to_host(s->vertex->vertexCellNeighbors, vcn, 3 * nv);
    to_host(s->vertex->cellVertexNum, cvn, nc);
    to_host(s->vertex->cell_vertices(), cv, nc * s->vertex->vmax());
    return 0;
}

int ref_vertex_set_positions(void *h, const double *vpos)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int nv = s->vertex->getNumberOfDegreesOfFreedom();
    std::vector<Dscalar2> p(nv);
    for (int i = 0; i < nv; ++i) p[i] = make_Dscalar2(vpos[2 * i], vpos[2 * i + 1]);
    s->vertex->setVertexPositions(p);
    return 0;
}

void ref_vertex_set_preferences(void *h, const double *pref)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int n = s->vertex->cells();
    std::vector<Dscalar2> p(n);
    for (int i = 0; i < n; ++i) p[i] = make_Dscalar2(pref[2 * i], pref[2 * i + 1]);
    s->vertex->setCellPreferences(p);
}

void ref_vertex_set_t1(void *h, double t) { reinterpret_cast<RefSystem *>(h)->vertex->setT1Threshold(t); }

double ref_vertex_forces(void *h, double *F, double *AP)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int nc = s->vertex->cells(), nv = s->vertex->getNumberOfDegreesOfFreedom();
    s->vertex->computeForces();
    to_host(s->vertex->returnForces(), reinterpret_cast<Dscalar2 *>(F), nv);
    to_host(s->vertex->returnAreaPeri(), reinterpret_cast<Dscalar2 *>(AP), nc);
    // the quadratic part (VertexQuadraticEnergyWithTension::computeEnergy is not implemented)
    return s->vertex->VertexQuadraticEnergy::computeEnergy();
}

// VertexQuadraticEnergyWithTension: cell types and one gamma (gammas == NULL) or an ntypes x ntypes
// matrix, tension on (computeVertexTensionForcesCPU)
void ref_vertex_set_tension(void *h, const int *types, double gamma, int ntypes, const double *gammas)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int nc = s->vertex->cells();
    std::vector<int> t(types, types + nc);
    s->vertex->setCellType(t);
    if (gammas) s->vertex->setSurfaceTension(std::vector<Dscalar>(gammas, gammas + (size_t)ntypes * ntypes));
    else s->vertex->setSurfaceTension(gamma);
    s->vertex->setUseSurfaceTension(true);
    s->vertex->dirty();
}

// Brownian timesteps (CPU branch, reproducible noise: two deviates per vertex, x then y)
int ref_vertex_brownian_run(void *h, int steps, double dt, double T, double mu)
{
    RefSystem *s = reinterpret_cast<RefSystem *>(h);
    int nv = s->vertex->getNumberOfDegreesOfFreedom();
    if (!s->sim) {
        auto bd = std::make_shared<brownianParticleDynamics>(nv);
        bd->setT(T);
        bd->setMu(mu);
        s->eom = bd;
        s->sim = std::make_shared<Simulation>();
        s->sim->setConfiguration(s->vertex);
        s->sim->addUpdater(bd, s->vertex);
        s->sim->setIntegrationTimestep(dt);
        s->sim->setCPUOperation(true);
        s->sim->setReproducible(true);
    }
    for (int t = 0; t < steps; ++t) s->sim->performTimestep();
    return 0;
}

// ---- Voronoi model with line tension: forces, A/P and energy of one state ---------------------
// gammas == NULL: one tension gamma for every pair of unlike types (setSurfaceTension(g));
// else an ntypes x ntypes matrix (setSurfaceTension(vector)). Returns computeEnergy().
double ref_voronoi_tension_forces(int n, const double *pos, const int *types, const double *pref, double gamma,
                                  int ntypes, const double *gammas, double *F, double *AP)
{
    RefVoronoiTension v(n, 1.0, 3.8);
    v.setCPU(true);
    std::vector<Dscalar2> p(n), ap(n);
    for (int i = 0; i < n; ++i) {
        p[i] = make_Dscalar2(pos[2 * i], pos[2 * i + 1]);
        ap[i] = make_Dscalar2(pref[2 * i], pref[2 * i + 1]);
    }
    v.setCellPositions(p);
    v.retriangulate();
    std::vector<int> t(types, types + n);
    v.setCellType(t);
    v.setCellPreferences(ap);
    if (gammas) v.setSurfaceTension(std::vector<Dscalar>(gammas, gammas + (size_t)ntypes * ntypes));
    else v.setSurfaceTension(gamma);
    v.setUseSurfaceTension(true);
    v.computeForces();
    to_host(v.returnForces(), reinterpret_cast<Dscalar2 *>(F), n);
    to_host(v.returnAreaPeri(), reinterpret_cast<Dscalar2 *>(AP), n);
    return v.computeEnergy();
}

}  // extern "C"
