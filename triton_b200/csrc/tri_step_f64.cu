// tri_step_f64.cu -- the step kernels instantiated for double.
#include "tri_step_launch.cuh"

namespace tri {
template int launch_step<double>(const StepArgs&, cudaStream_t, cudaEvent_t*);
template int launch_initial_dt<double>(const StepArgs&, cudaStream_t);
template void flux_occupancy<double>(int, int*);
template int launch_batch_step<double>(const BatchArgs&, cudaStream_t);
template int launch_batch_steps<double>(const BatchArgs&, MemberProgress*, int, int, cudaStream_t);
template int batch_steps_grid<double>(int);
template void batch_flux_occupancy<double>(int, int*);
template int prepare_kernels<double>();
}  // namespace tri
