// cellgpu_b200 -- C++ class API over the C ABI (include/cellgpu_b200.h).
//
// Keeps the reference's driver-facing classes and method names so that a program written against
// cellGPU's Simulation / VoronoiQuadraticEnergy (Voronoi2D) / VertexQuadraticEnergy /
// selfPropelledParticleDynamics / selfPropelledCellVertexDynamics / brownianParticleDynamics /
// EnergyMinimizerFIRE (inc/Simulation.h, inc/models/*.h, inc/updaters/*.h) compiles against this
// header with its include changed. Header-only; link with -lcellgpu_b200.
//
// Differences from the reference, by design:
//  * state is device-resident: returnPositions()/returnForces()/returnAreaPeri() copy to host
//    vectors on demand instead of handing out GPUArray references;
//  * the GPU is the only backend: setCPUOperation(true) throws;
//  * a failing call throws cellgpu::Error (the reference's HANDLE_ERROR throws std::exception).
#pragma once

#include <algorithm>
#include <cmath>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cellgpu_b200.h"

namespace cellgpu {

using Dscalar = double;
using Dscalar2 = double2;  // inc/std_include.h:47-60 with Dscalar = double
constexpr Dscalar PI = 3.14159265358979323846;

class Error : public std::runtime_error {
public:
    Error(int code, const std::string &what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int code)
{
    if (code != CG_OK) throw Error(code, cg_last_error_string());
}

// Seeded uniform positions in [0,L)^2, x then y per cell as Simple2DCell::setCellPositionsRandomly
// (src/models/Simple2DCell.cpp:85-100) draws them; SplitMix64 stream of the seed.
inline std::vector<Dscalar2> random_positions(int n, Dscalar L, unsigned long long seed)
{
    std::vector<Dscalar2> p(n);
    unsigned long long z = seed;
    auto next = [&z]() {
        z += 0x9E3779B97F4A7C15ull;
        unsigned long long x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int i = 0; i < n; ++i) {
        p[i].x = next() * L;
        p[i].y = next() * L;
    }
    return p;
}

// ---- models --------------------------------------------------------------------------------
class Simple2DModel {
public:
    virtual ~Simple2DModel()
    {
        if (sys_) cg_destroy(sys_);
    }
    Simple2DModel(const Simple2DModel &) = delete;
    Simple2DModel &operator=(const Simple2DModel &) = delete;

    cg_system *handle() const { return sys_; }
    virtual bool isVertexModel() const = 0;
    // order-independent (fixed-point) force sums: bit-identical forces and trajectories on reruns
    void setDeterministic(bool on) { check(cg_set_deterministic(sys_, on ? 1 : 0)); }
    virtual int getNumberOfDegreesOfFreedom() { return cg_num_dofs(sys_); }
    int getNumberOfCells() const { return Ncells; }

    void setCellPreferencesUniform(Dscalar A0, Dscalar P0)
    {
        std::vector<Dscalar2> ap(Ncells, make_double2(A0, P0));
        setCellPreferences(ap);
    }
    void setCellPreferences(std::vector<Dscalar2> &AreaPeriPreferences)
    {
        check(cg_set_cell_preferences(sys_, reinterpret_cast<const double *>(AreaPeriPreferences.data())));
    }
    void setModuliUniform(Dscalar newKA, Dscalar newKP) { check(cg_set_moduli(sys_, newKA, newKP)); }
    void setv0Dr(Dscalar v0new, Dscalar drnew)
    {
        std::vector<Dscalar2> m(Ncells, make_double2(v0new, drnew));
        check(cg_set_motility(sys_, reinterpret_cast<const double *>(m.data())));
    }
    void setCellMotility(std::vector<Dscalar> &v0s, std::vector<Dscalar> &drs)
    {
        std::vector<Dscalar2> m(Ncells);
        for (int i = 0; i < Ncells; ++i) m[i] = make_double2(v0s[i], drs[i]);
        check(cg_set_motility(sys_, reinterpret_cast<const double *>(m.data())));
    }
    void setCellDirectors(const std::vector<Dscalar> &theta) { check(cg_set_directors(sys_, theta.data())); }
    void setCellDirectorsRandomly(unsigned long long seed)
    {
        std::vector<Dscalar2> u = random_positions(Ncells, 1.0, seed ^ 0x5bd1e995ull);
        std::vector<Dscalar> th(Ncells);
        for (int i = 0; i < Ncells; ++i) th[i] = 2.0 * PI * u[i].x;
        setCellDirectors(th);
    }
    // device-noise keys of the model (RNG counters are the step and the local index)
    void setSeed(unsigned long long seed) { check(cg_set_seed(sys_, seed)); }

    virtual void computeForces() { check(cg_compute_forces(sys_)); }
    virtual void enforceTopology() { check(cg_enforce_topology(sys_)); }
    Dscalar computeEnergy()
    {
        computeForces();
        double E = 0.0;
        check(cg_get_energies(sys_, &E));
        return E;
    }
    std::vector<Dscalar2> returnPositions()
    {
        std::vector<Dscalar2> p(getNumberOfDegreesOfFreedom());
        check(cg_get_positions(sys_, reinterpret_cast<double *>(p.data())));
        return p;
    }
    std::vector<Dscalar2> returnForces()
    {
        std::vector<Dscalar2> f(getNumberOfDegreesOfFreedom());
        check(cg_get_forces(sys_, reinterpret_cast<double *>(f.data())));
        return f;
    }
    std::vector<Dscalar2> returnAreaPeri()
    {
        std::vector<Dscalar2> ap(Ncells);
        check(cg_get_area_perimeter(sys_, reinterpret_cast<double *>(ap.data())));
        return ap;
    }
    // mean and variance of the shape index q = P / sqrt(A) (Simple2DCell::reportq, reportVarq)
    Dscalar reportq()
    {
        std::vector<Dscalar2> ap = returnAreaPeri();
        double s = 0;
        for (auto &v : ap) s += v.y / std::sqrt(v.x);
        return s / Ncells;
    }
    Dscalar reportVarq()
    {
        std::vector<Dscalar2> ap = returnAreaPeri();
        double s = 0, s2 = 0;
        for (auto &v : ap) {
            double q = v.y / std::sqrt(v.x);
            s += q;
            s2 += q * q;
        }
        s /= Ncells;
        return s2 / Ncells - s * s;
    }
    Dscalar reportMeanP()
    {
        std::vector<Dscalar2> ap = returnAreaPeri();
        double s = 0;
        for (auto &v : ap) s += v.y;
        return s / Ncells;
    }
    long long counter(int i)
    {
        long long c[8] = {0};
        check(cg_counters(sys_, c, 8));
        return c[i];
    }

    int Ncells = 0;
    Dscalar L = 0.0;

protected:
    Simple2DModel() = default;
    cg_system *sys_ = nullptr;
};

// Voronoi (SPV) model: VoronoiQuadraticEnergy(n, A0, P0, reprod) of
// inc/models/voronoiQuadraticEnergy.h:20-22 (random positions in a box of side sqrt(n); reproducible
// runs use a fixed seed)
class VoronoiQuadraticEnergy : public Simple2DModel {
public:
    explicit VoronoiQuadraticEnergy(int n, bool reprod = false) : VoronoiQuadraticEnergy(n, 1.0, 3.8, reprod) {}
    VoronoiQuadraticEnergy(int n, Dscalar A0, Dscalar P0, bool reprod = false, int precision = CG_FP64)
    {
        Ncells = n;
        L = std::sqrt((double)n);
        double box[2] = {L, L};
        check(cg_voronoi_create(1, &n, box, 16, precision, &sys_));
        seed_ = reprod ? 13377ull : (unsigned long long)std::random_device{}();
        setSeed(seed_);
        setCellPositions(random_positions(n, L, seed_));
        setCellDirectorsRandomly(seed_);
        setCellPreferencesUniform(A0, P0);
        setv0Dr(0.05, 1.0);
    }
    bool isVertexModel() const override { return false; }
    void setCellPositions(const std::vector<Dscalar2> &newCellPositions)
    {
        check(cg_set_positions(sys_, reinterpret_cast<const double *>(newCellPositions.data())));
        check(cg_triangulate(sys_));
    }
    void globalTriangulationCGAL() { check(cg_triangulate(sys_)); }
    void setCPU(bool) { throw Error(CG_ERR_ARG, "cellgpu_b200 runs on the GPU only"); }
    // Delaunay neighbour rows (CCW), K entries per cell
    void getNeighbors(std::vector<int> &nn, std::vector<int> &nbr)
    {
        int K = cg_neighbor_capacity(sys_);
        nn.resize(Ncells);
        nbr.resize((size_t)Ncells * K);
        check(cg_get_topology(sys_, nn.data(), nbr.data()));
    }
    // particle exclusions (voronoiModelBase::setExclusions, src/models/voronoiModelBase.cpp:85-104):
    // excluded cells get v0 = Dr = 0 and, after every force evaluation, F = 0 with the computed
    // force kept as the external force
    void setExclusions(std::vector<int> &exes) { check(cg_set_exclusions(sys_, exes.data())); }
    void getExternalForces(std::vector<Dscalar2> &out)
    {
        out.resize(Ncells);
        check(cg_get_external_forces(sys_, reinterpret_cast<double *>(out.data())));
    }

private:
    unsigned long long seed_ = 0;
};
using Voronoi2D = VoronoiQuadraticEnergy;


// Vertex (AVM) model from the Delaunay dual of random cell positions:
// VertexQuadraticEnergy(n, A0, P0, reprod, runSPVToInitialize) of inc/models/vertexQuadraticEnergy.h:20
class VertexQuadraticEnergy : public Simple2DModel {
public:
    VertexQuadraticEnergy(int n, Dscalar A0, Dscalar P0, bool reprod = false, bool runSPVToInitialize = false)
    {
        if (runSPVToInitialize) throw Error(CG_ERR_ARG, "runSPVToInitialize is not supported");
        Ncells = n;
        L = std::sqrt((double)n);
        double box[2] = {L, L};
        check(cg_vertex_create(1, &n, box, 30, CG_FP64, &sys_));
        seed_ = reprod ? 13377ull : (unsigned long long)std::random_device{}();
        setSeed(seed_);
        std::vector<Dscalar2> cells = random_positions(n, L, seed_);
        check(cg_vertex_from_voronoi(sys_, reinterpret_cast<const double *>(cells.data())));
        setCellDirectorsRandomly(seed_);
        setCellPreferencesUniform(A0, P0);
        setv0Dr(0.05, 1.0);
        setT1Threshold(0.01);
    }
    bool isVertexModel() const override { return true; }
    void setT1Threshold(Dscalar t1t) { check(cg_set_t1_threshold(sys_, t1t)); }
    // vertices from the Delaunay dual of these cell positions (vertexModelBase::setCellsVoronoiTesselation)
    void setCellsVoronoiTesselation(const std::vector<Dscalar2> &cells)
    {
        check(cg_vertex_from_voronoi(sys_, reinterpret_cast<const double *>(cells.data())));
    }
    void setVertexPositions(const std::vector<Dscalar2> &v)
    {
        check(cg_set_positions(sys_, reinterpret_cast<const double *>(v.data())));
    }
    void setCPU(bool = true) { throw Error(CG_ERR_ARG, "cellgpu_b200 runs on the GPU only"); }

private:
    unsigned long long seed_ = 0;
};

// Line tension between cells of different types: setCellType, setSurfaceTension (one gamma, or a
// flattened symmetric ntypes x ntypes matrix) and setUseSurfaceTension of
// VoronoiQuadraticEnergyWithTension (inc/models/voronoiQuadraticEnergyWithTension.h:15-60) and
// VertexQuadraticEnergyWithTension (inc/models/vertexQuadraticEnergyWithTension.h). For the vertex
// model computeEnergy includes the tension, which the reference leaves unimplemented.
template <typename Model>
class WithTension : public Model {
public:
    template <typename... Args>
    explicit WithTension(Args &&...args) : Model(std::forward<Args>(args)...)
    {
        setCellType(std::vector<int>(this->Ncells, 0));
    }
    // Simple2DCell::setCellType
    void setCellType(const std::vector<int> &types) { check(cg_set_cell_types(this->sys_, types.data())); }
    void setUseSurfaceTension(bool use_tension)
    {
        Tension = use_tension;
        apply();
    }
    void setSurfaceTension(Dscalar g)
    {
        gamma = g;
        simpleTension = true;
        apply();
    }
    void setSurfaceTension(const std::vector<Dscalar> &gammas)
    {
        int n = (int)std::lround(std::sqrt((double)gammas.size()));
        if ((size_t)n * n != gammas.size()) throw Error(CG_ERR_ARG, "the tension matrix must be square");
        tensionMatrix = gammas;
        simpleTension = false;
        apply();
    }
    Dscalar getSurfaceTension() const { return gamma; }

private:
    void apply()
    {
        if (!Tension) check(cg_set_tension(this->sys_, 0.0));
        else if (simpleTension) check(cg_set_tension(this->sys_, gamma));
        else
            check(cg_set_tension_matrix(this->sys_, (int)std::lround(std::sqrt((double)tensionMatrix.size())),
                                        tensionMatrix.data()));
    }
    Dscalar gamma = 0.0;
    bool Tension = false, simpleTension = true;
    std::vector<Dscalar> tensionMatrix;
};
using VoronoiQuadraticEnergyWithTension = WithTension<VoronoiQuadraticEnergy>;
using VertexQuadraticEnergyWithTension = WithTension<VertexQuadraticEnergy>;

// ---- updaters ------------------------------------------------------------------------------
class updater {
public:
    virtual ~updater() = default;
    virtual void set2DModel(std::shared_ptr<Simple2DModel> model) { State = std::move(model); }
    virtual void setDeltaT(Dscalar dt) { deltaT = dt; }
    Dscalar getDeltaT() const { return deltaT; }
    virtual void Update(int n_steps = 1) { integrateEquationsOfMotion(n_steps); }
    virtual void integrateEquationsOfMotion(int n_steps = 1) = 0;

protected:
    std::shared_ptr<Simple2DModel> need()
    {
        if (!State) throw Error(CG_ERR_STATE, "updater has no model (set2DModel)");
        return State;
    }
    std::shared_ptr<Simple2DModel> State;
    Dscalar deltaT = 0.01;
};

// dr/dt = mu F + v0 n, dtheta/dt = noise (src/updaters/selfPropelledParticleDynamics.cpp:45-130);
// on a vertex model this is selfPropelledCellVertexDynamics
class selfPropelledParticleDynamics : public updater {
public:
    selfPropelledParticleDynamics() = default;
    explicit selfPropelledParticleDynamics(int) {}
    void setMu(Dscalar m) { mu = m; }
    Dscalar getMu() const { return mu; }
    void integrateEquationsOfMotion(int n_steps = 1) override
    {
        auto m = need();
        if (m->isVertexModel()) check(cg_vertex_spp_run(m->handle(), n_steps, deltaT, mu, nullptr));
        else check(cg_spp_run(m->handle(), n_steps, deltaT, mu, nullptr));
    }

protected:
    Dscalar mu = 1.0;
};

class selfPropelledCellVertexDynamics : public selfPropelledParticleDynamics {
public:
    selfPropelledCellVertexDynamics() = default;
    selfPropelledCellVertexDynamics(int, int) {}
};

// d = xi sqrt(2 dt T mu) + dt mu F (src/updaters/brownianParticleDynamics.cpp:46-109)
class brownianParticleDynamics : public updater {
public:
    brownianParticleDynamics() = default;
    explicit brownianParticleDynamics(int) {}
    void setT(Dscalar t) { T = t; }
    void setMu(Dscalar m) { mu = m; }
    void integrateEquationsOfMotion(int n_steps = 1) override
    {
        auto m = need();
        if (!m->isVertexModel()) throw Error(CG_ERR_ARG, "Brownian dynamics drives the vertex model");
        check(cg_brownian_run(m->handle(), n_steps, deltaT, mu, T, nullptr));
    }

private:
    Dscalar T = 0.0, mu = 1.0;
};

// FIRE (src/updaters/EnergyMinimizerFIRE2D.cpp), CPU conventions, defaults of :24-41
class EnergyMinimizerFIRE : public updater {
public:
    EnergyMinimizerFIRE() { initializeParameters(); }
    explicit EnergyMinimizerFIRE(std::shared_ptr<Simple2DModel> system)
    {
        initializeParameters();
        set2DModel(std::move(system));
    }
    void initializeParameters()
    {
        prm = {0.01, 0.1, 0.01 * 0.01, 1.05, 0.95, 0.99, 0.9, 1e-7, 5, 1000};
    }
    void setMaximumIterations(int maxIt) { prm.max_iterations = maxIt; }
    void setForceCutoff(Dscalar fc) { prm.force_cutoff = fc; }
    void setDeltaT(Dscalar dt) override
    {
        prm.dt = dt;
        prm.dt_min = dt * 0.01;
    }
    void setAlphaStart(Dscalar as) { prm.alpha_start = as; }
    void setDeltaTMax(Dscalar tmax) { prm.dt_max = tmax; }
    void setDeltaTInc(Dscalar dti) { prm.dt_inc = dti; }
    void setDeltaTDec(Dscalar dtc) { prm.dt_dec = dtc; }
    void setAlphaDec(Dscalar ad) { prm.alpha_dec = ad; }
    void setNMin(int nm) { prm.n_min = nm; }
    void minimize() { check(cg_fire_minimize(need()->handle(), &prm)); }
    void integrateEquationsOfMotion(int = 1) override { minimize(); }
    int getCurrentIterations()
    {
        int it = 0;
        double fm = 0, fn = 0;
        check(cg_fire_state(need()->handle(), &it, &fm, &fn));
        return it;
    }
    Dscalar getMaxForce()  // sqrt(max |F|^2) of the last iteration
    {
        int it = 0;
        double fm = 0, fn = 0;
        check(cg_fire_state(need()->handle(), &it, &fm, &fn));
        return fm;
    }

private:
    cg_fire_params prm{};
};

// ---- Simulation (inc/Simulation.h:18-87; performTimestep, src/Simulation.cpp:141-166) -------
class Simulation {
public:
    void setConfiguration(std::shared_ptr<Simple2DModel> config)
    {
        configuration = std::move(config);
        if (configuration && reproducible) configuration->setDeterministic(true);
    }
    void addUpdater(std::shared_ptr<updater> upd) { addUpdater(std::move(upd), configuration); }
    void addUpdater(std::shared_ptr<updater> upd, std::shared_ptr<Simple2DModel> config)
    {
        upd->set2DModel(config ? config : configuration);
        upd->setDeltaT(integrationTimestep);
        updaters.push_back(std::move(upd));
    }
    void clearUpdaters() { updaters.clear(); }
    void setIntegrationTimestep(Dscalar dt)
    {
        integrationTimestep = dt;
        for (auto &u : updaters) u->setDeltaT(dt);
    }
    void setCPUOperation(bool setcpu)
    {
        if (setcpu) throw Error(CG_ERR_ARG, "cellgpu_b200 runs on the GPU only");
    }
    // Reproducible runs (Simulation::setReproducible): besides fixed seeds, the configuration sums
    // its forces in an order-independent way, so reruns give bit-identical trajectories.
    void setReproducible(bool r)
    {
        reproducible = r;
        if (configuration) configuration->setDeterministic(r);
    }
    // re-sort the (Voronoi) configuration spatially every sp steps (src/Simulation.cpp:154-164)
    void setSortPeriod(int sp) { sortPeriod = sp; }
    void setCurrentTime(Dscalar t) { Time = t; }
    void setCurrentTimestep(int t) { integerTimestep = t; }
    void performTimestep() { performTimesteps(1); }
    // n steps of every updater back to back on the device (one graph replay per updater chunk)
    void performTimesteps(int n)
    {
        while (n > 0) {
            int chunk = n;
            if (sortPeriod > 0) chunk = std::min(n, sortPeriod - integerTimestep % sortPeriod);
            for (auto &u : updaters) u->Update(chunk);
            integerTimestep += chunk;
            Time += chunk * integrationTimestep;
            n -= chunk;
            if (sortPeriod > 0 && integerTimestep % sortPeriod == 0 && configuration &&
                !configuration->isVertexModel())
                check(cg_spatial_sort(configuration->handle()));
        }
    }

    int integerTimestep = 0;
    Dscalar Time = 0.0;
    Dscalar integrationTimestep = 0.01;
    int sortPeriod = -1;

private:
    std::shared_ptr<Simple2DModel> configuration;
    std::vector<std::shared_ptr<updater>> updaters;
    bool reproducible = false;
};

using SimulationPtr = std::shared_ptr<Simulation>;
using EOMPtr = std::shared_ptr<updater>;
using UpdaterPtr = std::shared_ptr<updater>;
using ForcePtr = std::shared_ptr<Simple2DModel>;

}  // namespace cellgpu
