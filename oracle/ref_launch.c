/*
 * Launchers for the reference's OpenCL kernels compiled as C (TEST
 * INFRASTRUCTURE ONLY).  Linked with binary_pursuit.cl (compiled through
 * clshim.h) into oracle/_ref/libbp_ref.so.  Each launch runs work-items
 * offset..offset+gsize-1 with a work-group size of 1.  Arguments arrive as an
 * array of 64-bit words in kernel-argument order: a buffer or local-memory
 * argument is its address, a scalar argument its value.  The prototypes
 * restate the kernel signatures of binary_pursuit.cl.
 *
 * bpref_launch runs the work-items one after another in global-id order.
 * bpref_launch_mt runs the work-items of the kernels whose work-items write
 * disjoint outputs -- compute_full_likelihood (one (window, template) each),
 * overlap_recheck_indices (one (a, b, t) item each; with a work-group size of
 * 1 every item is its own group and writes its own group result) and
 * get_adjusted_clips (one spike each) -- on several threads (OpenMP), each
 * thread with private copies of the local-memory arguments; the other kernels
 * read what neighbouring work-items write and stay in order.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
typedef unsigned int uint;
typedef unsigned char uchar;
_Thread_local size_t clshim_gid, clshim_lid, clshim_lsz = 1;

void compute_residual(float *, uint, uint, const float *, uint, uint, const uint *, const uint *, uint);                           /* .cl:57 */
void compute_full_likelihood(float *, uint, uint, const float *, uint, uint, const float *, const uint *, uint, float *);          /* .cl:255 */
void compute_template_maximum_likelihood(uint, uint, uint, const uint *, uint, uint *, uint *, float *, uchar *, uchar *,
                                         uint *, uint *, float *, const float *);                                                 /* .cl:350 */
void overlap_recheck_indices(float *, uint, uint, const float *, uint, uint, const uint *, uint, uint *, uint *, float *, uint,
                             float *, uint *, float *, uint *, const float *);                                                     /* .cl:444 */
void parse_overlap_recheck_indices(uint, uint, const uint *, uint, uint *, uint *, float *, uint *, uint *, float *, uint,
                                   const float *, float *, uint *, uchar *);                                                       /* .cl:657 */
void check_overlap_reassignments(uint, uint, const uint *, uint, uint *, uint *, uchar *, uint *, uint *, uchar *);              /* .cl:822 */
void binary_pursuit(uint, uint, uint, const float *, uint *, uint, const uint *, const uint *, const float *, uint *, uint *,
                    uint *, uint *, uchar *, uchar *);                                                                             /* .cl:918 */
void get_adjusted_clips(const float *, uint, uint, const float *, uint, uint, const uint *, const uint *, uint, float *);        /* .cl:1088 */

#define P(i, T) ((T)(uintptr_t)a[i])
#define U(i) ((uint)a[i])

/* One work-item of kernel `kernel` (ids follow the order of the .cl file). */
static int run_item(int kernel, uint64_t g, const uint64_t *a)
{
    clshim_lsz = 1;
    clshim_lid = 0;
    clshim_gid = (size_t)g;
    {
        switch (kernel) {
        case 0: compute_residual(P(0, float *), U(1), U(2), P(3, const float *), U(4), U(5), P(6, const uint *),
                                 P(7, const uint *), U(8)); break;
        case 1: compute_full_likelihood(P(0, float *), U(1), U(2), P(3, const float *), U(4), U(5), P(6, const float *),
                                        P(7, const uint *), U(8), P(9, float *)); break;
        case 2: compute_template_maximum_likelihood(U(0), U(1), U(2), P(3, const uint *), U(4), P(5, uint *), P(6, uint *),
                                                    P(7, float *), P(8, uchar *), P(9, uchar *), P(10, uint *),
                                                    P(11, uint *), P(12, float *), P(13, const float *)); break;
        case 3: overlap_recheck_indices(P(0, float *), U(1), U(2), P(3, const float *), U(4), U(5), P(6, const uint *), U(7),
                                        P(8, uint *), P(9, uint *), P(10, float *), U(11), P(12, float *), P(13, uint *),
                                        P(14, float *), P(15, uint *), P(16, const float *)); break;
        case 4: parse_overlap_recheck_indices(U(0), U(1), P(2, const uint *), U(3), P(4, uint *), P(5, uint *), P(6, float *),
                                              P(7, uint *), P(8, uint *), P(9, float *), U(10), P(11, const float *),
                                              P(12, float *), P(13, uint *), P(14, uchar *)); break;
        case 5: check_overlap_reassignments(U(0), U(1), P(2, const uint *), U(3), P(4, uint *), P(5, uint *), P(6, uchar *),
                                            P(7, uint *), P(8, uint *), P(9, uchar *)); break;
        case 6: binary_pursuit(U(0), U(1), U(2), P(3, const float *), P(4, uint *), U(5), P(6, const uint *),
                               P(7, const uint *), P(8, const float *), P(9, uint *), P(10, uint *), P(11, uint *),
                               P(12, uint *), P(13, uchar *), P(14, uchar *)); break;
        case 7: get_adjusted_clips(P(0, const float *), U(1), U(2), P(3, const float *), U(4), U(5), P(6, const uint *),
                                   P(7, const uint *), U(8), P(9, float *)); break;
        default: return -2;
        }
    }
    return 0;
}

int bpref_launch(int kernel, uint64_t offset, uint64_t gsize, uint64_t lsize, const uint64_t *a)
{
    if (lsize != 1) return -1;
    for (uint64_t g = offset; g < offset + gsize; g++)
        if (run_item(kernel, g, a)) return -2;
    return 0;
}

#define MAX_ARGS 32
/* local_bytes[i] > 0 marks argument i as local memory of that many bytes. */
int bpref_launch_mt(int kernel, uint64_t offset, uint64_t gsize, uint64_t lsize, const uint64_t *a,
                    int nargs, const uint64_t *local_bytes, int nthreads)
{
    if (lsize != 1 || nargs > MAX_ARGS) return -1;
    if (kernel != 1 && kernel != 3 && kernel != 7) return bpref_launch(kernel, offset, gsize, lsize, a);
    int bad = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        uint64_t args[MAX_ARGS];
        void *priv[MAX_ARGS] = {0};
        memcpy(args, a, (size_t)nargs * sizeof(uint64_t));
        for (int i = 0; i < nargs; i++)
            if (local_bytes[i]) {
                priv[i] = calloc((size_t)local_bytes[i] + 64, 1);
                if (!priv[i]) bad = 1;
                args[i] = (uint64_t)(uintptr_t)priv[i];
            }
#pragma omp barrier
        if (!bad) {
#pragma omp for schedule(dynamic, 64)
            for (long long g = (long long)offset; g < (long long)(offset + gsize); g++)
                run_item(kernel, (uint64_t)g, args);
        }
        for (int i = 0; i < nargs; i++) free(priv[i]);
    }
    return bad ? -3 : 0;
}
