/* Data-resident device types and memory helpers.
 * Replaces src/dev_type.h:9-101.  The enum keeps the reference's values.
 * This build is the GPU path only: DEV_TYPE_CUDA and DEV_TYPE_CUDA_MPI_DIRECT
 * both mean "pointers are device memory on the current CUDA device";
 * DEV_TYPE_HOST is rejected by the engines (there is no CPU fallback). */
#ifndef CA3DMM_DEV_TYPE_H
#define CA3DMM_DEV_TYPE_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include "ca3dmm_vmpi.h"

typedef enum {
    DEV_TYPE_HOST = 0,        /* CPU memory (rejected by the GPU engines) */
    DEV_TYPE_CUDA,            /* CUDA memory */
    DEV_TYPE_CUDA_MPI_DIRECT  /* CUDA memory (same as DEV_TYPE_CUDA here) */
} dev_type_t;

#ifdef __cplusplus
extern "C" {
#endif

/* src/dev_type.c:14-23: 1 if dev_type is a type the GPU engines accept. */
int is_dev_type_valid(dev_type_t dev_type);
/* src/dev_type.c:26-52: cudaMalloc for CUDA types, pinned host memory for HOST. */
void *dev_type_malloc(size_t bytes, dev_type_t dev_type);
/* src/dev_type.c:55-75 */
void dev_type_free(void *mem, dev_type_t dev_type);
/* src/dev_type.h:43-45 */
void dev_type_memset(void *mem, int value, size_t bytes, dev_type_t dev_type);
/* src/dev_type.c:105-130: cudaMemcpy with the direction taken from the types. */
void dev_type_memcpy(void *dst, const void *src, size_t bytes, dev_type_t dst_dev_type,
                     dev_type_t src_dev_type);
/* src/dev_type.c:133-156: copy a row-major nrow x ncol block (dt_size 4 or 8)
 * between device buffers with the batched pack kernel. */
void dev_type_copy_mat_blk(size_t dt_size, const int nrow, const int ncol, const void *src,
                           const int lds, void *dst, const int ldd, dev_type_t dev_type);

#ifdef __cplusplus
}
#endif

/* src/dev_type.h:76-101.  For the GPU types only the device work buffer is
 * allocated (workbuf_h stays NULL): the engines never stage through host. */
#define MALLOC_ATTACH_WORKBUF(attach_func, free_func, engine, dev_type, workbuf_bytes, workbuf_h, \
                              workbuf_d)                                                       \
    do {                                                                                       \
        workbuf_h = NULL;                                                                      \
        workbuf_d = NULL;                                                                      \
        if ((engine) == NULL) break;                                                           \
        if ((dev_type) == DEV_TYPE_HOST) {                                                     \
            workbuf_h = dev_type_malloc(workbuf_bytes, DEV_TYPE_HOST);                         \
        } else {                                                                               \
            workbuf_d = dev_type_malloc(workbuf_bytes, DEV_TYPE_CUDA);                         \
            if (workbuf_d == NULL && (workbuf_bytes) > 0) {                                    \
                fprintf(stderr, "[ERROR] %s, %d: Allocate CUDA workbuf failed\n", __FILE__,   \
                        __LINE__);                                                             \
                free_func(&engine);                                                            \
                break;                                                                         \
            }                                                                                  \
        }                                                                                      \
        attach_func(engine, workbuf_h, workbuf_d);                                             \
    } while (0)

#endif
