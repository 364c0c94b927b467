/* Empty stand-in: capi.c includes this header but uses nothing from it. */
#ifndef TM_REF_SHIM_IUSET_H
#define TM_REF_SHIM_IUSET_H
#endif
