/*
 * stubs.c -- HDF5 archive entry points of the reference (h5io.F90).  The
 * archive is not part of this library; the symbols exist so that callers
 * that bind them up front (python/fteik3d.py:99-103) still load, and every
 * call reports failure.
 */
#include <stdio.h>

static int h5_unavailable(const char *who)
{
    fprintf(stderr, "%s: HDF5 archives are not available in this library\n", who);
    return 1;
}

int fteik_h5io_initializeF(const char *fileName)
{
    (void)fileName;
    return h5_unavailable("fteik_h5io_initializeF");
}

int fteik_h5io_finalizeF(void) { return h5_unavailable("fteik_h5io_finalizeF"); }

int fteik_h5io_writeLevelSchedulesF(void)
{
    return h5_unavailable("fteik_h5io_writeLevelSchedulesF");
}

int fteik_h5io_writeVelocityModelF(const char *velName)
{
    (void)velName;
    return h5_unavailable("fteik_h5io_writeVelocityModelF");
}

int fteik_h5io_writeTravelTimesF(const char *ttName)
{
    (void)ttName;
    return h5_unavailable("fteik_h5io_writeTravelTimesF");
}
