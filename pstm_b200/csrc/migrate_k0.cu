// Instantiations of the gather kernel for traveltime kind 0.
#include "migrate_dispatch.cuh"
namespace pstm {
template cudaError_t launch_migrate<0>(const KParams &, const KParams *, int, bool, int, const Launch &);
}
