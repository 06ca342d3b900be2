// Instantiations of the gather kernel for traveltime kind 1.
#include "migrate_dispatch.cuh"
namespace pstm {
template cudaError_t launch_migrate<1>(const KParams &, const KParams *, int, bool, int, const Launch &);
}
