// Timing harness in the manner of the reference's voronoi.cpp: a Voronoi monolayer driven by
// self-propelled particle dynamics through the class API; prints the time per step.
// Options: -n cells, -t timed steps, -i initialisation steps, -e dt, -p p0, -v v0.
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "cellgpu.hpp"

using namespace cellgpu;

int main(int argc, char **argv)
{
    int numpts = 200, tSteps = 5, initSteps = 1, c;
    Dscalar dt = 0.01, p0 = 3.8, v0 = 0.1;
    while ((c = getopt(argc, argv, "n:t:i:e:p:v:")) != -1) {
        switch (c) {
        case 'n': numpts = atoi(optarg); break;
        case 't': tSteps = atoi(optarg); break;
        case 'i': initSteps = atoi(optarg); break;
        case 'e': dt = atof(optarg); break;
        case 'p': p0 = atof(optarg); break;
        case 'v': v0 = atof(optarg); break;
        default: fprintf(stderr, "usage: %s [-n cells] [-t steps] [-i init] [-e dt] [-p p0] [-v v0]\n", argv[0]);
                 return 1;
        }
    }
    try {
        auto spp = std::make_shared<selfPropelledParticleDynamics>(numpts);
        auto spv = std::make_shared<VoronoiQuadraticEnergy>(numpts, 1.0, 4.0, true);
        spv->setCellPreferencesUniform(1.0, p0);
        spv->setv0Dr(v0, 1.0);
        auto sim = std::make_shared<Simulation>();
        sim->setConfiguration(spv);
        sim->addUpdater(spp, spv);
        sim->setIntegrationTimestep(dt);
        sim->setCPUOperation(false);
        sim->setReproducible(true);
        printf("starting initialization\n");
        sim->performTimesteps(initSteps);
        printf("Finished with initialization\ncurrent q = %f\n", spv->reportq());
        long long repairs0 = spv->counter(2);
        auto t1 = std::chrono::steady_clock::now();
        sim->performTimesteps(tSteps);
        spv->computeEnergy();  // synchronises the system's stream
        auto t2 = std::chrono::steady_clock::now();
        double steptime = std::chrono::duration<double>(t2 - t1).count() / tSteps;
        printf("timestep ~ %g per frame; energy %f\n", steptime, spv->computeEnergy());
        printf("%f\n", spv->reportq());
        printf("number of local topology updates per cell per tau = %g\n",
               (spv->counter(2) - repairs0) * (1.0 / numpts) * (1.0 / tSteps / dt));
    } catch (const Error &e) {
        fprintf(stderr, "cellgpu error %d: %s\n", e.code(), e.what());
        return 1;
    }
    return 0;
}
