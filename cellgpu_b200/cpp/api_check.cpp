// Drives the C++ class API on deterministic states and prints the results as one JSON line, so a
// test can compare them with the Python API on the same states. States: R2 quasi-random cell
// positions, golden-ratio directors; seeds of reproducible models (13377).
#include <cstdio>
#include <cstdlib>

#include "cellgpu.hpp"

using namespace cellgpu;

static std::vector<Dscalar2> r2_points(int n, double L)
{
    const double a1 = 0.7548776662466927, a2 = 0.5698402909980532;
    std::vector<Dscalar2> p(n);
    for (int i = 0; i < n; ++i) {
        double x = 0.5 + a1 * (i + 1), y = 0.5 + a2 * (i + 1);
        p[i] = make_double2((x - std::floor(x)) * L, (y - std::floor(y)) * L);
    }
    return p;
}

static std::vector<Dscalar> golden_angles(int n)
{
    std::vector<Dscalar> t(n);
    for (int i = 0; i < n; ++i) {
        double x = 0.5 + 0.6180339887498949 * i;
        t[i] = 2.0 * PI * (x - std::floor(x));
    }
    return t;
}

static void print_head(const char *name, const std::vector<Dscalar2> &v, int k)
{
    printf("\"%s\": [", name);
    for (int i = 0; i < k; ++i) printf("%s%.17g, %.17g", i ? ", " : "", v[i].x, v[i].y);
    printf("]");
}

int main(int argc, char **argv)
{
    int nv = argc > 1 ? atoi(argv[1]) : 400;
    int nx = argc > 2 ? atoi(argv[2]) : 240;
    try {
        // Voronoi model, SPP through Simulation, then FIRE
        auto spv = std::make_shared<VoronoiQuadraticEnergy>(nv, 1.0, 3.8, true);
        spv->setCellPositions(r2_points(nv, spv->L));
        spv->setCellDirectors(golden_angles(nv));
        spv->setCellPreferencesUniform(1.0, 3.8);
        double E0 = spv->computeEnergy();
        std::vector<Dscalar2> F0 = spv->returnForces();
        spv->setv0Dr(0.1, 1.0);
        auto spp = std::make_shared<selfPropelledParticleDynamics>(nv);
        auto sim = std::make_shared<Simulation>();
        sim->setConfiguration(spv);
        sim->addUpdater(spp, spv);
        sim->setIntegrationTimestep(0.01);
        sim->setCPUOperation(false);
        sim->setReproducible(true);
        for (int i = 0; i < 50; ++i) sim->performTimestep();
        std::vector<Dscalar2> P1 = spv->returnPositions();
        auto fire = std::make_shared<EnergyMinimizerFIRE>(spv);
        fire->setForceCutoff(1e-10);
        fire->setMaximumIterations(10000);
        fire->minimize();
        double Ef = spv->computeEnergy();

        // vertex model from the dual of the same kind of state, Brownian + T1, then FIRE
        auto avm = std::make_shared<VertexQuadraticEnergy>(nx, 1.0, 3.8, true);
        avm->setCellsVoronoiTesselation(r2_points(nx, avm->L));
        avm->setT1Threshold(0.04);
        double V0 = avm->computeEnergy();
        auto bd = std::make_shared<brownianParticleDynamics>(2 * nx);
        bd->setT(1e-3);
        auto sim2 = std::make_shared<Simulation>();
        sim2->setConfiguration(avm);
        sim2->addUpdater(bd, avm);
        sim2->setIntegrationTimestep(0.005);
        sim2->performTimesteps(50);
        std::vector<Dscalar2> VP = avm->returnPositions();
        auto fire2 = std::make_shared<EnergyMinimizerFIRE>(avm);
        fire2->setForceCutoff(1e-10);
        fire2->setMaximumIterations(10000);
        fire2->minimize();
        double Vf = avm->computeEnergy();

        // line tension: alternating types, one gamma, then a symmetric 2 x 2 matrix
        auto ten = std::make_shared<VoronoiQuadraticEnergyWithTension>(nv, 1.0, 3.8, true);
        ten->setCellPositions(r2_points(nv, ten->L));
        std::vector<int> types(nv);
        for (int i = 0; i < nv; ++i) types[i] = i % 2;
        ten->setCellType(types);
        ten->setSurfaceTension(0.2);
        ten->setUseSurfaceTension(true);
        double T1 = ten->computeEnergy();
        std::vector<Dscalar2> TF1 = ten->returnForces();
        ten->setSurfaceTension(std::vector<Dscalar>{0.0, 0.35, 0.35, 0.0});
        double T2 = ten->computeEnergy();

        printf("{\"tension\": {\"E_simple\": %.17g, \"E_matrix\": %.17g, ", T1, T2);
        print_head("F_simple", TF1, 4);
        printf("}, ");
        printf("\"voronoi\": {\"n\": %d, \"E0\": %.17g, ", nv, E0);
        print_head("F0", F0, 4);
        printf(", ");
        print_head("P_spp", P1, 4);
        printf(", \"fire_iterations\": %d, \"fire_fmax\": %.17g, \"E_fire\": %.17g, \"q\": %.17g}, ",
               fire->getCurrentIterations(), fire->getMaxForce(), Ef, spv->reportq());
        printf("\"vertex\": {\"n\": %d, \"E0\": %.17g, ", nx, V0);
        print_head("P_brownian", VP, 4);
        printf(", \"t1_flips\": %lld, \"fire_iterations\": %d, \"fire_fmax\": %.17g, \"E_fire\": %.17g}}\n",
               avm->counter(5), fire2->getCurrentIterations(), fire2->getMaxForce(), Vf);
    } catch (const Error &e) {
        fprintf(stderr, "cellgpu error %d: %s\n", e.code(), e.what());
        return 1;
    }
    return 0;
}
