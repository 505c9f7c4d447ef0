// Instantiations of the thread-per-run kernel family.
#include "sim_serial.cuh"

namespace csmc {
template int serial_launch_one<false, false>(const SimParams &, int, int, size_t, void *);
template int serial_launch_one<false, true>(const SimParams &, int, int, size_t, void *);
template int serial_launch_one<true, false>(const SimParams &, int, int, size_t, void *);
template int serial_launch_one<true, true>(const SimParams &, int, int, size_t, void *);
template int serial_occupancy_one<false, false>(int, size_t, int *);
template int serial_occupancy_one<false, true>(int, size_t, int *);
template int serial_occupancy_one<true, false>(int, size_t, int *);
template int serial_occupancy_one<true, true>(int, size_t, int *);
}  // namespace csmc
