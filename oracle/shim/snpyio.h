/*
 * Stand-in for the two SimpleNpyIO calls SimpleTCSolver makes (oracle build
 * only; SimpleNpyIO is an empty submodule in the reference, .gitmodules:5-8).
 * Signatures follow the call sites src/fileio.c:194 and :251: the dtype
 * string carries its quotes ("'<f8'", src/fileio.c:20-22), shape and dtype
 * returned by the reader are heap memory the caller frees.
 */
#if !defined(TCREF_SHIM_SNPYIO_H)
#define TCREF_SHIM_SNPYIO_H

#include <stdio.h>
#include <stdbool.h>
#include <stddef.h>

int snpyio_r_header(
    size_t * ndims,
    size_t ** shape,
    char ** dtype,
    bool * is_fortran_order,
    FILE * fp,
    size_t * header_size
);

int snpyio_w_header(
    const size_t ndims,
    const size_t * shape,
    const char dtype[],
    const bool is_fortran_order,
    FILE * fp,
    size_t * header_size
);

#endif // TCREF_SHIM_SNPYIO_H
