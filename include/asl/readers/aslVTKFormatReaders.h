/* readers/aslVTKFormatReaders.h -- ASL header name of the LBGK path; readSurface is in
 * aslb_asl_io.hpp (over the C ABI of libaslb.so, aslb.h). */
#ifndef ASLB_FACADE_READERS_ASLVTKFORMATREADERS_H
#define ASLB_FACADE_READERS_ASLVTKFORMATREADERS_H
#include "../aslb_asl_std.hpp"
#endif
