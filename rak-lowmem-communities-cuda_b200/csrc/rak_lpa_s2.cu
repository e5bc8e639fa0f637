// Instantiates the persistent LPA kernel for 2 sketch slot(s) (separate unit: parallel build).
#include "rak_lpa.cuh"

namespace rak {
template cudaError_t launch_lpa_slots<2>(const LpaArgs &, int, bool, bool, cudaStream_t, int *);
template cudaError_t resolve_lpa_slots<2>(int, bool, bool, bool, bool, const void **, int *);
}
