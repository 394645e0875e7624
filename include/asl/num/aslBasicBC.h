/* num/aslBasicBC.h -- ASL header name of the LBGK path; the classes and functions are in
 * aslb_asl.hpp (over the C ABI of libaslb.so, aslb.h). */
#ifndef ASLB_FACADE_NUM_ASLBASICBC_H
#define ASLB_FACADE_NUM_ASLBASICBC_H
#include "../aslb_asl_std.hpp"
#endif
