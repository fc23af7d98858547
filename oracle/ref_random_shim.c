/*
 * The reference's own Gaussian random fill and element-weight error kernel,
 * compiled from its sources (TEST INFRASTRUCTURE ONLY, built into
 * oracle/_ref/liboskar_ref.so by `make -C oracle ref`):
 *
 *  - mem/src/oskar_mem_random_gaussian.c is included as it is, so that its
 *    CPU fill loops (mem_random_gaussian_{float,double}: Random123 Philox
 *    4x32-10 from the reference's extern/Random123, then Box-Muller from
 *    math/private_random_helpers.h) can be called on plain arrays. Its
 *    oskar_Mem entry point is never called; the container and device
 *    accessors it references are stubbed below so that the library loads.
 *  - telescope/station/define_evaluate_element_weights_errors.h is
 *    instantiated as the CPU kernel.
 *
 * ref_element_weights_errors_{d,f} chain the two the way
 * oskar_evaluate_element_weights_errors.c:19-110 does on the CPU.
 */
#include "mem/src/oskar_mem_random_gaussian.c"
#include "utility/oskar_kernel_macros.h"
#include "utility/oskar_vector_types.h"
#include "telescope/station/define_evaluate_element_weights_errors.h"

OSKAR_ELEMENT_WEIGHTS_ERR(k_weights_errors_f, float, float2)
OSKAR_ELEMENT_WEIGHTS_ERR(k_weights_errors_d, double, double2)

void ref_random_gaussian_d(unsigned int n, double* data, unsigned int seed,
        unsigned int c1, unsigned int c2, unsigned int c3, double std)
{
    mem_random_gaussian_double(n, data, seed, c1, c2, c3, std);
}

void ref_random_gaussian_f(unsigned int n, float* data, unsigned int seed,
        unsigned int c1, unsigned int c2, unsigned int c3, float std)
{
    mem_random_gaussian_float(n, data, seed, c1, c2, c3, std);
}

void ref_element_weights_errors_d(int n, const double* gain,
        const double* gain_error, const double* phase,
        const double* phase_error, unsigned int seed, int time_index,
        int station_id, double* errors)
{
    mem_random_gaussian_double(2 * (unsigned int) n, errors, seed,
            (unsigned int) time_index, (unsigned int) station_id,
            0x12345678u, 1.0);
    k_weights_errors_d(n, gain, gain_error, phase, phase_error,
            (double2*) errors);
}

void ref_element_weights_errors_f(int n, const float* gain,
        const float* gain_error, const float* phase,
        const float* phase_error, unsigned int seed, int time_index,
        int station_id, float* errors)
{
    mem_random_gaussian_float(2 * (unsigned int) n, errors, seed,
            (unsigned int) time_index, (unsigned int) station_id,
            0x12345678u, 1.0f);
    k_weights_errors_f(n, gain, gain_error, phase, phase_error,
            (float2*) errors);
}

/* Never called: oskar_mem_random_gaussian() references them. */
size_t oskar_mem_length(const oskar_Mem* mem) { (void) mem; return 0; }
int oskar_mem_location(const oskar_Mem* mem) { (void) mem; return 0; }
int oskar_mem_precision(const oskar_Mem* mem) { (void) mem; return 0; }
int oskar_mem_is_complex(const oskar_Mem* mem) { (void) mem; return 0; }
int oskar_mem_is_matrix(const oskar_Mem* mem) { (void) mem; return 0; }
void* oskar_mem_buffer(oskar_Mem* mem) { (void) mem; return 0; }
float* oskar_mem_float(oskar_Mem* mem, int* status)
{ (void) mem; (void) status; return 0; }
double* oskar_mem_double(oskar_Mem* mem, int* status)
{ (void) mem; (void) status; return 0; }
void oskar_device_check_local_size(int location, unsigned int dim,
        size_t local_size[3])
{ (void) location; (void) dim; (void) local_size; }
void oskar_device_launch_kernel(const char* name, int location,
        int num_dims, size_t local_size[3], size_t global_size[3],
        size_t num_args, const oskar_Arg* arg,
        size_t num_local_args, const size_t* arg_size_local, int* status)
{
    (void) name; (void) location; (void) num_dims; (void) local_size;
    (void) global_size; (void) num_args; (void) arg; (void) num_local_args;
    (void) arg_size_local; (void) status;
}
