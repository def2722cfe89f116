/* Test infrastructure only.  The reference's example executables divide their domain over
 * omp_get_num_devices() devices and need at least one; built for the CPU (no offload target)
 * libgomp reports none and the target regions run on the host.  This definition, linked into
 * the executable, reports one device, so each driver runs its one-device configuration. */
int omp_get_num_devices(void) { return 1; }
