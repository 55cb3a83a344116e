// Stand-in for green-utils' MPI context: the ranks gpu_kernel.cpp:27-37 reads.  Declarations only.
#pragma once
namespace green::utils {
struct mpi_context {
  int global_rank = 0;
  int node_rank = 0;
};
mpi_context& context();
}  // namespace green::utils
