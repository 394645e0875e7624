// Host-side checks of the ASL C++ facade (no GPU): vectors, blocks,
// distance functions and maps, parameters, and the VTK writer on a plain
// data container. Prints one "key value..." line per check for
// tests/test_facade_cpu.py; exits non-zero on a failed assertion.
#include <aslDataInc.h>
#include <aslGeomInc.h>
#include <acl/aclGenerators.h>
#include <math/aslTemplates.h>
#include <utilities/aslParametersManager.h>
#include <writers/aslVTKFormatWriters.h>

#include <cstdio>
#include <cstring>

using asl::AVec;
using asl::makeAVec;

#define EXPECT(c)                                             \
  do {                                                        \
    if (!(c)) {                                               \
      std::fprintf(stderr, "failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                               \
    }                                                         \
  } while (0)

int main(int argc, char* argv[]) {
  asl::ApplicationParametersManager pm("facade_host", "1.0");
  asl::Parameter<AVec<int>> size(makeAVec(12, 10, 8), "size", "cells");
  asl::Parameter<double> radius(3.0, "radius", "cylinder radius");
  asl::Parameter<std::string> out(std::string("facade_host"), "output", "vti prefix");
  pm.load(argc, argv);

  // vectors: a * b is the scalar product
  AVec<> a = makeAVec(1., 2., 3.), b = makeAVec(4., 5., 6.);
  EXPECT(a * b == 32.);
  EXPECT((a + b)[2] == 9. && (b - a)[0] == 3. && (2. * a)[1] == 4. && (a / 2.)[2] == 1.5);
  EXPECT(asl::crossProduct(a, b) == makeAVec(-3., 6., -3.));
  EXPECT(asl::minComponent(b) == 4. && asl::maxComponent(b) == 6. && asl::productOfElements(makeAVec(2, 3, 4)) == 24);

  // blocks: z-fastest flattening, far corner, offsets
  asl::Block block(size.v(), 0.5, makeAVec(1., 2., 3.));
  EXPECT(block.c2i(makeAVec(1, 2, 3)) == (1 * size.v()[1] + 2) * size.v()[2] + 3);
  EXPECT(block.getBPosition() == makeAVec(1. + 0.5 * (size.v()[0] - 1), 2. + 0.5 * (size.v()[1] - 1),
                                          3. + 0.5 * (size.v()[2] - 1)));
  asl::Block g = asl::offset(block, 1);
  EXPECT(g.getSize() == size.v() + AVec<int>(3, 2) && g.position == makeAVec(0.5, 1.5, 2.5));

  // lattices
  EXPECT(asl::d3q19().q == 19 && asl::d3q19().vectors[1] == makeAVec(1, 0, 0));
  double wsum = 0;
  for (double w : asl::d3q27().quasiparticlesCoefs) wsum += w;
  EXPECT(std::fabs(wsum - 1.0) < 1e-12);

  // a normalised cylinder map on the ghosted block, FP32 and FP64 containers
  auto df = asl::normalize(asl::generateDFCylinderInf(radius.v(), makeAVec(0., 0., 1.), makeAVec(3., 4., 0.)), 0.5);
  auto m32 = asl::generateDataContainerACL_SP<float>(block, 1, 1u);
  auto m64 = asl::generateDataContainerACL_SP<double>(block, 1, 1u);
  asl::initData(m32, df);
  asl::initData(m64, df);
  // union with a sphere, intersection, inversion
  auto u = asl::generateDFSphere(1.0, makeAVec(5., 5., 5.)) | asl::generateDFPlane(makeAVec(0., 0., 1.), makeAVec(0., 0., 4.));
  EXPECT(u->getDistance(5., 5., 5.) == -1.0 && u->getDistance(5., 5., 0.) == -4.0);
  EXPECT((-u)->getDistance(5., 5., 5.) == 1.0);
  EXPECT((asl::generateDFSphere(1.0, makeAVec(0., 0., 0.)) & asl::generateDFSphere(1.0, makeAVec(1., 0., 0.)))
             ->getDistance(0., 0., 0.) == 0.0);
  auto cyl = asl::generateDFCylinder(1.0, makeAVec(0., 0., 2.), makeAVec(0., 0., 0.));
  EXPECT(cyl->getDistance(0., 0., 0.) == -1.0 && cyl->getDistance(0., 0., 3.) == 2.0);
  // an empty operand leaves the other one (unions built up from nothing)
  asl::SPDistanceFunction none;
  EXPECT((none | u) == u && (u & none) == u);
  auto inb = asl::generateDFInBlock(asl::Block(makeAVec(10, 10, 10), 1.0), 0);
  EXPECT(inb->getDistance(4.5, 4.5, 4.5) == 5.0 && inb->getDistance(-1., 4.5, 4.5) == -0.5 &&
         inb->getDistance(4.5, 4.5, 10.) == -0.5);

  // the FP32 map as raw floats (compared with the Python rasteriser)
  std::printf("map32");
  for (float v : m32->floats()) {
    unsigned int bits;
    std::memcpy(&bits, &v, 4);
    std::printf(" %08x", bits);
  }
  std::printf("\n");
  const std::vector<double>& v64 = m64->values();
  double maxdiff = 0;
  for (size_t i = 0; i < v64.size(); ++i) maxdiff = std::max(maxdiff, std::fabs(v64[i] - m32->values()[i]));
  std::printf("map64_vs_map32 %.3e\n", maxdiff);

  // a vector container and the writer
  auto vec = asl::generateDataContainerACL_SP<float>(block, 3, 1u);
  std::vector<double>& vv = vec->values();
  const size_t n = vec->cells();
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) vv[c * n + i] = double(i) + 0.25 * c;
  asl::WriterVTKXML writer(out.v());
  writer.addScalars("map", *m32);
  writer.addVector("vec", *vec);
  writer.write();
  writer.write();
  std::printf("writes %u\n", writer.getNumOfWrites());
  std::printf("params %d %d %d %.3f %s\n", size.v()[0], size.v()[1], size.v()[2], radius.v(), out.v().c_str());

  // constant values per component, and the parameters directory
  auto cv = asl::generateDataContainerACL_SP<float>(asl::Block(makeAVec(3, 2, 2)), 3, 1u);
  asl::initData(cv, makeAVec(1.5, -2., 0.25));
  const std::vector<double>& cvv = cv->values();
  const size_t cn = cv->cells();
  EXPECT(cvv[0] == 1.5 && cvv[cn - 1] == 1.5 && cvv[cn] == -2. && cvv[3 * cn - 1] == 0.25);
  asl::initData(cv, 0.75);
  EXPECT(cv->values()[2 * cn] == 0.75);
  std::printf("dir %s\n", pm.getDir().c_str());

  // errors carry ASL's prefix
  try {
    asl::offset(asl::Block(makeAVec(1, 1, 1)), -2);
    return 1;
  } catch (const std::logic_error& e) {
    std::printf("error %s\n", e.what());
  }
  return 0;
}
