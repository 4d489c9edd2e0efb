/*
 * Build configuration of the B200 supermesh library.  Replaces the header
 * CMake generates from include/libsupermesh.h.in in libsupermesh
 * (firedrakeproject/libsupermesh include/libsupermesh.h.in:23-35); the
 * library is always built in double precision, so
 * LIBSUPERMESH_DOUBLE_PRECISION is always defined (libsupermesh-c.h would
 * otherwise silently switch c_kind to float).
 */
#ifndef LIBSUPERMESH_LIBSUPERMESH_H
#define LIBSUPERMESH_LIBSUPERMESH_H

#define LIBSUPERMESH_VERSION_MAJOR 1
#define LIBSUPERMESH_VERSION_MINOR 0
#define LIBSUPERMESH_VERSION_PATCH 1
#define LIBSUPERMESH_VERSION "1.0.1+b200"
#define LIBSUPERMESH_GIT_REVISION "unknown"

#define LIBSUPERMESH_DOUBLE_PRECISION

/* Marks this build as the GPU implementation (no counterpart upstream). */
#define LIBSUPERMESH_B200 1

#endif
