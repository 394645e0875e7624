/* num/aslLBGK.h -- ASL header name of the LBGK path; the classes and functions are in
 * aslb_asl.hpp (over the C ABI of libaslb.so, aslb.h). */
#ifndef ASLB_FACADE_NUM_ASLLBGK_H
#define ASLB_FACADE_NUM_ASLLBGK_H
#include "../aslb_asl_std.hpp"
#endif
