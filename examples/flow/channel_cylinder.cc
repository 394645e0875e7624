// channel_cylinder.cc -- the canonical laminar case of the LBGK path, written
// against ASL's C++ API as its flow examples use it (ASL project:
// examples/flow/flow.cc:70-134): a D3Q19 channel of 128 x 64 x 64 cells in
// FP32, a cylinder of radius 8 along z through (32, 32), inlet velocity 0.05
// at X0, pressure 1 at XE, no-slip Y/Z walls, viscosity 0.01 (tau = 0.53),
// fluid at rest at the start, 1000 steps. Prints the drag and lift on the
// cylinder (the surface-force field summed in FP64) and writes density,
// velocity, map and force field to <output>_0.vti.
//
// Build (from the repository root, after the library is built):
//   g++ -std=c++17 -O2 -I include/asl -I include examples/flow/channel_cylinder.cc
//       -L asl_b200 -laslb -Wl,-rpath,$PWD/asl_b200 -o channel_cylinder
#include <utilities/aslParametersManager.h>
#include <aslDataInc.h>
#include <math/aslTemplates.h>
#include <aslGeomInc.h>
#include <acl/aclGenerators.h>
#include <writers/aslVTKFormatWriters.h>
#include <num/aslLBGK.h>
#include <num/aslLBGKBC.h>
#include <utilities/aslTimer.h>

#include <cstdio>

typedef float FlT;
typedef asl::UValue<double> Param;

using asl::AVec;
using asl::makeAVec;

int main(int argc, char* argv[]) {
  asl::ApplicationParametersManager appParamsManager("channel_cylinder", "1.0");
  asl::Parameter<AVec<int>> size(makeAVec(128, 64, 64), "size", "interior cells");
  asl::Parameter<unsigned int> steps(1000u, "steps", "time steps");
  asl::Parameter<std::string> output(std::string("channel_cylinder"), "output", "output file prefix");
  appParamsManager.load(argc, argv);

  Param dx(1.);
  Param nu(.01);

  asl::Block block(size.v(), dx.v());
  auto cylinder(asl::normalize(asl::generateDFCylinderInf(8., makeAVec(0., 0., 1.), makeAVec(32., 32., 0.)), dx.v()));
  auto cylinderMap(asl::generateDataContainerACL_SP<FlT>(block, 1, 1u));
  asl::initData(cylinderMap, cylinder);

  asl::SPLBGK lbgk(new asl::LBGK(block, acl::generateVEConstant(FlT(nu.v())), &asl::d3q19()));
  lbgk->init();
  asl::SPLBGKUtilities lbgkUtil(new asl::LBGKUtilities(lbgk));
  lbgkUtil->initF(acl::generateVEConstant(.0, .0, .0));

  std::vector<asl::SPNumMethod> bc;
  bc.push_back(asl::generateBCConstantVelocity(lbgk, makeAVec(0.05, 0., 0.), {asl::X0}));
  bc.push_back(asl::generateBCConstantPressure(lbgk, 1., {asl::XE}));
  bc.push_back(asl::generateBCNoSlip(lbgk, {asl::Y0, asl::YE, asl::Z0, asl::ZE}));
  bc.push_back(asl::generateBCNoSlip(lbgk, cylinderMap));
  auto forceField(asl::generateDataContainerACL_SP<FlT>(block, 3, 1u));
  auto computeForce(asl::generateComputeSurfaceForce(lbgk, forceField, cylinderMap));
  asl::initAll(bc);
  computeForce->init();

  asl::Timer timer;
  timer.start();
  for (unsigned int i = 1; i <= steps.v(); ++i) {
    lbgk->execute();
    asl::executeAll(bc);
  }
  computeForce->execute();
  timer.stop();

  // drag and lift: the force field over the block, summed in FP64
  const std::vector<double>& f = forceField->values();
  const size_t n = forceField->cells();
  double F[3] = {0, 0, 0};
  for (int c = 0; c < 3; ++c)
    for (size_t k = 0; k < n; ++k) F[c] += f[c * n + k];

  asl::WriterVTKXML writer(output.v());
  writer.addScalars("map", *cylinderMap);
  writer.addScalars("rho", *lbgk->getRho());
  writer.addVector("v", *lbgk->getVelocity());
  writer.addVector("force", *forceField);
  writer.write();

  std::printf("steps %u drag %.9e lift_y %.9e lift_z %.9e\n", steps.v(), F[0], F[1], F[2]);
  std::printf("Real Time = %g; Processor Time = %g; Processor Load = %g%%\n", timer.realTime(),
              timer.processorTime(), timer.processorLoad() * 100);
  return 0;
}
