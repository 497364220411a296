// tri_step_f32.cu -- the step kernels instantiated for float.
#include "tri_step_launch.cuh"

namespace tri {
template int launch_step<float>(const StepArgs&, cudaStream_t, cudaEvent_t*);
template int launch_initial_dt<float>(const StepArgs&, cudaStream_t);
template void flux_occupancy<float>(int, int*);
template int launch_batch_step<float>(const BatchArgs&, cudaStream_t);
template int launch_batch_steps<float>(const BatchArgs&, MemberProgress*, int, int, cudaStream_t);
template int batch_steps_grid<float>(int);
template void batch_flux_occupancy<float>(int, int*);
template int prepare_kernels<float>();
}  // namespace tri
