// hadros_trace_fast.cu — the trace kernel with the fast geodesic arithmetic
// (hadros_trace_kernel.cuh: geo_rhs_fast), compiled with FMA contraction.
#include "hadros_trace_kernel.cuh"

namespace hadros {

int launch_trace_fast(const TraceArgs& args, int precision, int n_sm, void* stream, std::string& err)
{
    return launch_variant<1>(args, precision, n_sm, static_cast<cudaStream_t>(stream), err);
}

int prepare_trace_fast(const TraceArgs& args, int precision, int n_sm, int blocks_per_sm, LaunchCfg& cfg,
                       std::string& err)
{
    return prepare_variant<1>(args, precision, n_sm, blocks_per_sm, cfg, err);
}

int launch_trace_prepared_fast(const TraceArgs& args, int precision, const LaunchCfg& cfg, void* stream,
                               std::string& err)
{
    return launch_prepared_variant<1>(args, precision, cfg, static_cast<cudaStream_t>(stream), err);
}

int launch_path_transfer_fast(const TraceArgs& args, int precision, int n_sm, void* stream, std::string& err)
{
    return launch_paths<1>(args, precision, n_sm, static_cast<cudaStream_t>(stream), err);
}

}  // namespace hadros
