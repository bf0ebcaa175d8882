/*
 * PolyPtr / ConstPolyPtr: the C-ABI handle for every polynomial argument.
 *
 * Byte-identical to the reference's structs (core/src/common/iter/src/iter.cuh:12-26) and to
 * the Rust #[repr(C)] twins (core/src/poly_ptr.rs:4-19): element i of the view lives at
 * data[(offset + i) % whole_len]; a non-zero rotate r turns into offset = len - r and then
 * requires offset == 0 and len == whole_len (iter.cuh:308-327).  Elements are 32-byte BN254
 * Fr values (8 little-endian u32 limbs, Montgomery form).  whole_len == 0 means len.
 *
 * Where the reference asserts on a malformed view, the functions of this library return
 * cudaErrorInvalidValue instead.
 */
#ifndef ZKP_POLY_PTR_H
#define ZKP_POLY_PTR_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct PolyPtr {
    unsigned int *ptr;
    size_t len;
    size_t rotate;
    size_t offset;
    size_t whole_len;
} PolyPtr;

typedef struct ConstPolyPtr {
    const unsigned int *ptr;
    size_t len;
    size_t rotate;
    size_t offset;
    size_t whole_len;
} ConstPolyPtr;

#ifdef __cplusplus
}
#endif
#endif
