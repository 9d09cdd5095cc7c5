// NVTX ranges around the library's public calls and host-side stages, so that a
// profiler (ncu --nvtx, Nsight Systems) attributes device work to them. NVTX v3
// is header-only: with no tool attached a range costs a pointer check.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace rnb {

struct TraceRange {
	explicit TraceRange(const char *name) { nvtxRangePushA(name); }
	~TraceRange() { nvtxRangePop(); }
	TraceRange(const TraceRange &) = delete;
	TraceRange &operator=(const TraceRange &) = delete;
};

} // namespace rnb
