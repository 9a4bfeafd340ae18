/*
 * Build-time stand-in for the reference's pconfig.h (Patmol pconfig.h:1-20),
 * force-included ahead of every reference source by oracle/Makefile while
 * _PCONFIG_H_ is predefined, so the reference's own pconfig.h becomes a no-op.
 *
 * Only the scratch directory changes: the reference hard-codes an absolute
 * cluster path (pconfig.h:5-6).  Here the ERI files go to the process's
 * working directory, so every run must use a directory of its own
 * (file names are <rank><fileno><basename>, erifs.c:25-41).
 * TMPDIR_LEN counts the terminating NUL because erifs.c:36 copies it with
 * strncpy and then strncat()s onto the result.
 *
 * Test infrastructure only: nothing in the product includes this file.
 */
#ifndef PATREF_PCONFIG_OVERRIDE_H
#define PATREF_PCONFIG_OVERRIDE_H
#include "config.h"

#define TMPDIR_NAME "./"
#define TMPDIR_LEN 3
#define MAXFILESIZE 1048576*1024
#define MAXL 5
#define MAXORB (1<<15)

#ifndef inline
#ifndef __inline__
#define inline
#else
#define inline __inline__
#endif
#endif

#endif
