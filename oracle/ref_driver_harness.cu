// ref_driver_harness.cu -- test infrastructure only: the reference's OWN filter
// driver loop, particle_filter() of src/partfilt/cuda/pf_generic_soa.cu:686-1302
// with the robot-arm model (src/models/robotarm/cuda/pf_model_soa.cuh), built
// with its CUDA MTGP32 generator (-DMTGP: mtgp32-cuda.cu, mtgp32-cuda-common.cu,
// mtgp32-fast.c and the 11213 parameter table) and -DDEBUG_ESTIMATE (it then
// prints each step's best particle and error and, at the end, "N m t
// mean-error").  Built by oracle/build_ref_driver.sh straight from the
// reference tree (its main() renamed, the legacy cutil.h replaced by
// oracle/cutil_shim/cutil.h) into oracle/_ref/; nothing of the reference is
// committed.
//
// The reference seeds its 120 MTGP32 streams with gettimeofday()'s
// microseconds (mtgp32-cuda-common.cu:43-47, stream i: seed + i + 1); the
// build routes gettimeofday to ref_fixed_gettimeofday below, so a run is
// reproducible and the engine can run the same streams (its
// PF_RNG_REFLAYOUT with 120 streams, the CUDA kernel's mask and that seed).
#include <fcntl.h>
#include <sys/time.h>
#include <unistd.h>

static unsigned g_ref_seed_usec = 0;

extern "C" int ref_fixed_gettimeofday(struct timeval* __restrict tv, void* __restrict) noexcept
{
    tv->tv_sec = 0;
    tv->tv_usec = (suseconds_t)g_ref_seed_usec;
    return 0;
}

#include "pf_generic_soa.cu"
#include "mtgp/mtgp32-cuda.cu"
#include "mtgp/mtgp32-cuda-common.cu"

// Runs the reference driver on a trace file with the MTGP32 seed `seed`
// (0 <= seed < 1e6, the microseconds it would have read), its standard
// output redirected to out_path.  Returns the driver's return value.
extern "C" int ref_particle_filter(int num_particles, int num_blocks, int num_transfer, float resampling_freq,
                                   const char* input_file, unsigned seed, const char* out_path)
{
    g_ref_seed_usec = seed;
    fflush(stdout);
    const int saved = dup(1);
    const int fd = open(out_path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (saved < 0 || fd < 0) return -1;
    dup2(fd, 1);
    close(fd);
    const int rc = particle_filter(num_particles, num_blocks, num_transfer, resampling_freq, input_file);
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    return rc;
}
