// readSurface through ASL's C++ API (include/asl): the three overloads on an
// STL file given as the first argument; each map is printed as its internal
// block (size, position, dx) and its FP32 values in hex, for comparison with
// the Python reader, which drives the same library calls.
#include <cstdio>
#include <cstring>
#include <string>

#include <aslGeomInc.h>
#include <readers/aslVTKFormatReaders.h>

using asl::makeAVec;

static void dump(const char* name, const asl::SPDataWithGhostNodesACLData& d) {
  const asl::Block& b = d->getInternalBlock();
  std::printf("%s %d %d %d %.17g %.17g %.17g %.17g", name, b.getSize()[0], b.getSize()[1], b.getSize()[2],
              b.position[0], b.position[1], b.position[2], b.dx);
  for (double v : d->values()) {
    const float f = float(v);
    unsigned int bits;
    std::memcpy(&bits, &f, 4);
    std::printf(" %08x", bits);
  }
  std::printf("\n");
}

int main(int argc, char* argv[]) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: facade_surface file.stl\n");
    return 2;
  }
  const std::string file = argv[1];
  asl::Block bl(makeAVec(24, 16, 12), 0.5, makeAVec(-2., -1., 0.5));
  dump("block", asl::readSurface(file, bl));
  dump("spacing", asl::readSurface(file, 0.5));
  dump("offsets", asl::readSurface(file, 0.5, .5, .25, 0., 1., 1., .5));
  try {
    asl::readSurface(file + ".obj", 0.5);
  } catch (const std::logic_error& e) {
    std::printf("error %s\n", e.what());
  }
  return 0;
}
