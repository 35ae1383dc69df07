// TEST INFRASTRUCTURE ONLY -- link stubs for the reference's GPU kernel callers (its .cu files
// are not compiled for the oracle). The CPU branch the oracle runs never calls them; if one is
// reached, the process stops with a message instead of running unbuilt GPU code.
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include "std_include.h"
#include "indexer.h"
#include "gpubox.h"

static bool cg_ref_gpu_stub(const char *name)
{
    fprintf(stderr, "reference GPU path %s is not built into the oracle\n", name);
    abort();
}

bool gpu_avm_force_sets(int*, double2*, double4*, double2*, double2*, double2*, int, double, double) { return cg_ref_gpu_stub("gpu_avm_force_sets"); }
bool gpu_avm_sum_force_sets(double2*, double2*, int) { return cg_ref_gpu_stub("gpu_avm_sum_force_sets"); }
bool gpu_brownian_eom_integration(double2*, double2*, curandStateXORWOW*, int, double, double, double) { return cg_ref_gpu_stub("gpu_brownian_eom_integration"); }
bool gpu_compute_cell_list(double2*, unsigned int*, int*, int, int&, int, int, double, gpubox&, Index2D&, Index2D&, int*) { return cg_ref_gpu_stub("gpu_compute_cell_list"); }
bool gpu_compute_voronoi_geometry(double2*, double2*, int*, int*, double2*, double4*, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_compute_voronoi_geometry"); }
bool gpu_displacement_velocity_verlet(double2*, double2*, double2*, double, int) { return cg_ref_gpu_stub("gpu_displacement_velocity_verlet"); }
bool gpu_dot_Dscalar2_vectors(double2*, double2*, double*, int) { return cg_ref_gpu_stub("gpu_dot_Dscalar2_vectors"); }
bool gpu_force_sets(double2*, double2*, double2*, int2*, int*, double2*, double4*, double2*, int2*, double, double, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_force_sets"); }
bool gpu_initialize_RNG_array(curandStateXORWOW*, int, int, int) { return cg_ref_gpu_stub("gpu_initialize_RNG_array"); }
bool gpu_move_degrees_of_freedom(double2*, double2*, double, int, gpubox&) { return cg_ref_gpu_stub("gpu_move_degrees_of_freedom"); }
bool gpu_move_degrees_of_freedom(double2*, double2*, int, gpubox&) { return cg_ref_gpu_stub("gpu_move_degrees_of_freedom"); }
bool gpu_parallel_reduction(double*, double*, double*, int, int) { return cg_ref_gpu_stub("gpu_parallel_reduction"); }
bool gpu_spp_eom_integration(double2*, double2*, double2*, double2*, double*, curandStateXORWOW*, int, double, int, double) { return cg_ref_gpu_stub("gpu_spp_eom_integration"); }
bool gpu_sum_force_sets(double2*, double2*, int*, int, Index2D&) { return cg_ref_gpu_stub("gpu_sum_force_sets"); }
bool gpu_sum_force_sets_with_exclusions(double2*, double2*, double2*, int*, int*, int, Index2D&) { return cg_ref_gpu_stub("gpu_sum_force_sets_with_exclusions"); }
bool gpu_test_circumcenters(int*, int3*, int, double2*, unsigned int*, int*, int, int, int, double, gpubox&, Index2D&, Index2D&, int*) { return cg_ref_gpu_stub("gpu_test_circumcenters"); }
bool gpu_update_velocity(double2*, double2*, double, int) { return cg_ref_gpu_stub("gpu_update_velocity"); }
bool gpu_update_velocity_FIRE(double2*, double2*, double, double, int) { return cg_ref_gpu_stub("gpu_update_velocity_FIRE"); }
bool gpu_vm_flip_edges(int*, double2*, int*, int*, int*, int*, int*, int4*, gpubox&, Index2D&, int, int) { return cg_ref_gpu_stub("gpu_vm_flip_edges"); }
bool gpu_vm_geometry(double2*, int*, int*, int*, double2*, double4*, double2*, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_vm_geometry"); }
bool gpu_vm_get_cell_positions(double2*, double2*, int*, int*, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_vm_get_cell_positions"); }
bool gpu_vm_parse_multiple_flips(int*, int*, int*, int*, int*, int*, int*, int*, int4*, Index2D&, int) { return cg_ref_gpu_stub("gpu_vm_parse_multiple_flips"); }
bool gpu_vm_test_edges_for_T1(double2*, int*, int*, int*, int*, int*, gpubox&, double, int, int, int*, Index2D&) { return cg_ref_gpu_stub("gpu_vm_test_edges_for_T1"); }
bool gpu_zero_array(int*, int) { return cg_ref_gpu_stub("gpu_zero_array"); }
bool gpu_zero_array(unsigned int*, int) { return cg_ref_gpu_stub("gpu_zero_array"); }
bool gpu_zero_velocity(double2*, int) { return cg_ref_gpu_stub("gpu_zero_velocity"); }
bool gpu_VoronoiTension_force_sets(double2*, double2*, double2*, int2*, int*, double2*, double4*, double2*, int2*, int*, double*, Index2D&, double, double, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_VoronoiTension_force_sets"); }
bool gpu_VoronoiSimpleTension_force_sets(double2*, double2*, double2*, int2*, int*, double2*, double4*, double2*, int2*, int*, double, double, double, int, Index2D&, gpubox&) { return cg_ref_gpu_stub("gpu_VoronoiSimpleTension_force_sets"); }
