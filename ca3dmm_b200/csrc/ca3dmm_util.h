/* Internal host helpers: the reference's print and environment-variable
 * conventions (src/utils.h:26-83), kept so logs and knobs read the same. */
#ifndef CA3DMM_UTIL_H
#define CA3DMM_UTIL_H

#include <stdio.h>
#include <stdlib.h>

#define INFO_PRINTF(fmt, ...)                                                              \
    do {                                                                                   \
        fprintf(stdout, "[INFO] %s, %d: " fmt, __FILE__, __LINE__, ##__VA_ARGS__);         \
        fflush(stdout);                                                                    \
    } while (0)
#define WARNING_PRINTF(fmt, ...)                                                           \
    do {                                                                                   \
        fprintf(stderr, "[WARNING] %s, %d: " fmt, __FILE__, __LINE__, ##__VA_ARGS__);      \
        fflush(stderr);                                                                    \
    } while (0)
#define ERROR_PRINTF(fmt, ...)                                                             \
    do {                                                                                   \
        fprintf(stderr, "[ERROR] %s, %d: " fmt, __FILE__, __LINE__, ##__VA_ARGS__);        \
        fflush(stderr);                                                                    \
    } while (0)

/* Integer knob from the environment: out-of-range values fall back to the
 * default (src/utils.h:71-83 semantics). */
#define GET_ENV_INT_VAR(var, env_str, var_str, default_val, min_val, max_val)              \
    do {                                                                                   \
        char *env_str_p = getenv(env_str);                                                 \
        if (env_str_p != NULL) {                                                           \
            var = atoi(env_str_p);                                                         \
            if (var < (min_val) || var > (max_val)) var = (default_val);                   \
            INFO_PRINTF("Overriding parameter %s: %d (default) --> %d (runtime)\n", var_str, \
                        (int) (default_val), (int) var);                                   \
        } else {                                                                           \
            var = (default_val);                                                           \
        }                                                                                  \
    } while (0)

/* Evaluate a CUDA runtime call; on failure print where and why and return
 * CA3DMM_ECUDA from the enclosing function. */
#define CA3DMM_CUDA_TRY(call)                                                              \
    do {                                                                                   \
        cudaError_t err_ = (call);                                                         \
        if (err_ != cudaSuccess) {                                                         \
            ERROR_PRINTF("%s failed: %s\n", #call, cudaGetErrorString(err_));              \
            return CA3DMM_ECUDA;                                                           \
        }                                                                                  \
    } while (0)

static inline long long ca3dmm_round_up(long long x, long long a) { return (x + a - 1) / a * a; }

double ca3dmm_wtime_sec(void);

#endif
