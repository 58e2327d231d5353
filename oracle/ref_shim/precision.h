#ifndef _PRECISION_H_
#define _PRECISION_H_
#include <stdint.h>
typedef double Float;
typedef double IFloat;
typedef uint64_t Pointer;
#endif
