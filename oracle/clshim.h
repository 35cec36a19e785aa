/*
 * OpenCL C -> C99 shim (TEST INFRASTRUCTURE ONLY).  Force-included when the
 * reference's unmodified spikesorting_fullpursuit/kernels/binary_pursuit.cl is
 * compiled as C for the CPU (oracle/Makefile, target `ref`).  Every kernel runs
 * with a work-group size of 1, one work-item after another in global-id order
 * (see ref_launch.c), so barrier() is a no-op and __local data is private.
 */
#ifndef FBP_CLSHIM_H
#define FBP_CLSHIM_H
#include <stddef.h>
#include <stdint.h>
#define __kernel
#define __global
#define __local
#define __private
#define __constant const
#define CLK_LOCAL_MEM_FENCE 0
#define CLK_GLOBAL_MEM_FENCE 0
extern _Thread_local size_t clshim_gid;
extern _Thread_local size_t clshim_lid;
extern _Thread_local size_t clshim_lsz;
#define get_global_id(d) (clshim_gid)
#define get_local_id(d) (clshim_lid)
#define get_local_size(d) (clshim_lsz)
#define barrier(f) ((void)0)
#define atomic_add(p, v) __atomic_fetch_add((p), (v), __ATOMIC_SEQ_CST)
#endif
