#ifndef INCLUDED_CONFIG_H_
#define INCLUDED_CONFIG_H_
#define NOARCH 0
#define QCDOC 1
#define QCDSP 2
#define BGL 3
#define BGP 4
#define BGQ 5
#define TARGET NOARCH
#define CPS_FLOAT_ALIGN
#define CWDPREFIX(A) A
#define CAST_AWAY_CONST(x) ( const_cast<char*>(x) )
#define GLOBALSUM_TYPE double
#define CPS_END_NAMESPACE }
#define CPS_START_NAMESPACE namespace cps {
#define USING_NAMESPACE_CPS using namespace cps;
#define CPS_NAMESPACE cps
#define COMMS_DATASIZE (sizeof(double))
#define HAVE_STDINT_H 1
#define HAVE_INT64_T 1
#define HAVE_UINT64_T 1
#define HAVE_POSIX_MEMALIGN 1
#define HAVE_MALLOC_H 1
#endif
