/* Replacement for SuperLU 6.0.1's CMake-generated superlu_config.h.
 * Test infrastructure only: used to compile the vendored SuperLU sources of
 * the reference for the oracle's reference build (oracle/_ref).
 * 32-bit sparse indices, COLAMD enabled, METIS disabled - the same choices the
 * reference's CMake build makes (CMakeLists.txt:20-21, enable_internal_blaslib). */
#ifndef SUPERLU_CONFIG_H
#define SUPERLU_CONFIG_H
#define HAVE_COLAMD 1
typedef int int_t;
#endif
