/*
 * scl_core.h — core C ABI of the B200 diffusion libraries
 * (libscl_<f32|f64>_<i32|i64>.so).
 *
 * Replaces scl/binding/c_api/core/core.h:39-187 of scl-core. Types, error codes
 * and function signatures are identical, so code written against scl-core's
 * core.h compiles and links against these libraries unchanged.
 *
 * Like scl-core, the element types are chosen per library variant: define
 * SCL_USE_FLOAT32 / SCL_USE_FLOAT64 and SCL_USE_INT32 / SCL_USE_INT64 before
 * including this header to match the library you link (defaults: float64,
 * int64, as in core.h:79-111).
 */
#ifndef SCL_B200_CORE_H
#define SCL_B200_CORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCL_C_API_VERSION_MAJOR 1
#define SCL_C_API_VERSION_MINOR 0
#define SCL_C_API_VERSION_PATCH 0

#if defined(__GNUC__) || defined(__clang__)
#define SCL_EXPORT __attribute__((visibility("default")))
#else
#define SCL_EXPORT
#endif

/* core.h:56 — runtime version string. */
SCL_EXPORT const char* scl_get_version(void);
/* core.h:59 — build configuration, e.g. "float32+int32+cuda-sm_100a". */
SCL_EXPORT const char* scl_get_build_config(void);

/* core.h:65-73 — opaque handles. */
typedef struct scl_sparse_matrix scl_sparse_matrix;
typedef struct scl_dense_matrix scl_dense_matrix;
typedef scl_sparse_matrix* scl_sparse_t;
typedef scl_dense_matrix* scl_dense_t;

/* core.h:79-111 — element types by variant. */
#if defined(SCL_USE_FLOAT32)
typedef float scl_real_t;
#define SCL_REAL_TYPE_NAME "float32"
#else
typedef double scl_real_t;
#define SCL_REAL_TYPE_NAME "float64"
#endif

#if defined(SCL_USE_INT32)
typedef int32_t scl_index_t;
#define SCL_INDEX_TYPE_NAME "int32"
#else
typedef int64_t scl_index_t;
#define SCL_INDEX_TYPE_NAME "int64"
#endif

typedef size_t scl_size_t;
typedef int scl_bool_t;
#define SCL_TRUE 1
#define SCL_FALSE 0

/* core.h:124-166 — error codes (stable values). */
typedef int32_t scl_error_t;
#define SCL_OK 0
#define SCL_ERROR_UNKNOWN 1
#define SCL_ERROR_INTERNAL 2
#define SCL_ERROR_OUT_OF_MEMORY 3
#define SCL_ERROR_NULL_POINTER 4
#define SCL_ERROR_INVALID_ARGUMENT 10
#define SCL_ERROR_DIMENSION_MISMATCH 11
#define SCL_ERROR_DOMAIN_ERROR 12
#define SCL_ERROR_RANGE_ERROR 13
#define SCL_ERROR_INDEX_OUT_OF_BOUNDS 14
#define SCL_ERROR_TYPE_ERROR 20
#define SCL_ERROR_TYPE_MISMATCH 21
#define SCL_ERROR_IO_ERROR 30
#define SCL_ERROR_FILE_NOT_FOUND 31
#define SCL_ERROR_PERMISSION_DENIED 32
#define SCL_ERROR_READ_ERROR 33
#define SCL_ERROR_WRITE_ERROR 34
#define SCL_ERROR_UNREGISTERED_POINTER 35
#define SCL_ERROR_BUFFER_NOT_FOUND 36
#define SCL_ERROR_NOT_IMPLEMENTED 40
#define SCL_ERROR_FEATURE_UNAVAILABLE 41
#define SCL_ERROR_NUMERICAL_ERROR 50
#define SCL_ERROR_DIVISION_BY_ZERO 51
#define SCL_ERROR_OVERFLOW 52
#define SCL_ERROR_UNDERFLOW 53
#define SCL_ERROR_CONVERGENCE_ERROR 54

/* core.h:168-187 — thread-local error state. */
SCL_EXPORT const char* scl_get_last_error(void);
SCL_EXPORT scl_error_t scl_get_last_error_code(void);
SCL_EXPORT void scl_clear_error(void);
SCL_EXPORT scl_bool_t scl_is_ok(scl_error_t code);
SCL_EXPORT scl_bool_t scl_is_error(scl_error_t code);

#ifdef __cplusplus
}
#endif
#endif /* SCL_B200_CORE_H */
