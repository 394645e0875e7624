/* aslb_asl_std.hpp -- ASL's acl headers put namespace std into the global
 * scope (src/acl/aclMath/aclVectorOfElementsDef.h:31, src/acl/aclMath/
 * aclMathAlg.h:30), and every ASL header that includes them passes that on:
 * ASL's example programs use cout, endl and vector unqualified. The thin
 * headers standing for those ASL headers include this file, so the programs
 * compile unchanged; aslb_asl.hpp itself stays free of it. */
#ifndef ASLB_ASL_STD_HPP
#define ASLB_ASL_STD_HPP
#include "aslb_asl_io.hpp"
using namespace std;
#endif
