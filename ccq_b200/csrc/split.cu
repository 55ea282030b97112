// Split-precision GETT (placeholder until the tcgen05 kernel lands).
#include <stdexcept>
#include "split.cuh"
namespace ccqb {
void split_reserve(SplitWorkspace &, SplitSizes, int) { throw std::runtime_error("split precision not built"); }
void split_free(SplitWorkspace &) {}
int split_gett(SplitWorkspace &, const GettArgs &, int, int, int, cudaStream_t) { throw std::runtime_error("split precision not built"); }
int split_launch_count(const GettArgs &, int) { return 0; }
}
