/*
 * fteik/fteik_fortran.h -- the reference's C include path
 * (include/fteik/fteik_fortran.h), kept so that C callers written against
 * the reference build unchanged with -I<this repository>/include and link
 * libfteik_shared.so from fteik_b200/lib.
 *
 * Every declaration lives in ../fteik_b200.h: the reference's prototypes with
 * their drift from the Fortran BIND(C) interfaces corrected, the ordering
 * constants, and this library's additions.
 */
#ifndef FTEIK_FORTRAN_H__
#define FTEIK_FORTRAN_H__
#include "../fteik_b200.h"
#endif
