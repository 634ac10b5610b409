/* Project-written stand-in (TEST INFRASTRUCTURE ONLY); nothing is needed from it. */
#ifndef ORACLE_SHIM_GSL_ERRNO_H
#define ORACLE_SHIM_GSL_ERRNO_H
#endif
