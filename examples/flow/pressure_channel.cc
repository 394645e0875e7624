// pressure_channel.cc -- a pressure-driven D3Q15 channel around a cylinder
// across it, written with the API calls of ASL's flow example (ASL project:
// examples/flow/flow.cc:53-144): a formula-backed obstacle map, pressure
// conditions on X0 and XE, no-slip walls and map, the visualisation condition
// on the velocity, a VTK writer and the timer. Sizes and values are this
// program's own: 96 x 32 x 32 cells in FP32, viscosity 0.02, pressures 1.02
// and 0.98, a cylinder of radius 4 along y through (24, *, 16).
//
// Build as channel_cylinder.cc. Options: --steps N, --output prefix,
// --every N (output period), --device N.
#include <utilities/aslParametersManager.h>
#include <aslDataInc.h>
#include <math/aslTemplates.h>
#include <aslGeomInc.h>
#include <acl/aclGenerators.h>
#include <writers/aslVTKFormatWriters.h>
#include <num/aslLBGK.h>
#include <num/aslLBGKBC.h>
#include <utilities/aslTimer.h>
#include <acl/aclUtilities.h>

#include <iostream>

typedef float FlT;
typedef asl::UValue<double> Param;

using asl::AVec;
using asl::makeAVec;

int main(int argc, char* argv[]) {
  asl::ApplicationParametersManager appParamsManager("pressure_channel", "1.0");
  asl::Parameter<unsigned int> steps(200u, "steps", "time steps");
  asl::Parameter<unsigned int> every(100u, "every", "output period");
  asl::Parameter<std::string> output(std::string("pressure_channel"), "output", "output file prefix");
  appParamsManager.load(argc, argv);

  Param dx(1.);
  Param dt(1.);
  Param nu(.02);
  Param nuNum(nu.v() * dt.v() / dx.v() / dx.v());
  AVec<int> size(makeAVec(96, 32, 32));
  auto gSize(dx.v() * AVec<>(size));

  asl::Block block(size, dx.v());
  auto obstacle(asl::generateDFCylinderInf(.125 * gSize[1], makeAVec(0., 1., 0.), makeAVec(.25 * gSize[0], 0., .5 * gSize[2])));
  auto obstacleMap(asl::generateDataContainer_SP(block, obstacle, 1u, acl::typeToTypeID<FlT>()));
  auto obstacleMapMem(asl::generateDataContainerACL_SP<FlT>(block, 1, 1u));
  asl::initData(obstacleMapMem, obstacle);

  asl::SPLBGK lbgk(new asl::LBGK(block, acl::generateVEConstant(FlT(nuNum.v())), &asl::d3q15()));
  lbgk->init();
  asl::SPLBGKUtilities lbgkUtil(new asl::LBGKUtilities(lbgk));
  lbgkUtil->initF(acl::generateVEConstant(.0, .0, .0));

  std::vector<asl::SPNumMethod> bc;
  std::vector<asl::SPNumMethod> bcVis;
  bc.push_back(asl::generateBCConstantPressure(lbgk, 1.02, {asl::X0}));
  bc.push_back(asl::generateBCConstantPressure(lbgk, 0.98, {asl::XE}));
  bc.push_back(generateBCNoSlip(lbgk, {asl::Y0, asl::YE, asl::Z0, asl::ZE}));
  bc.push_back(generateBCNoSlip(lbgk, obstacleMap));
  bcVis.push_back(generateBCNoSlipVel(lbgk, obstacleMap));
  initAll(bc);
  initAll(bcVis);

  asl::Timer timer;
  asl::WriterVTKXML writer(output.v());
  writer.addScalars("map", *obstacleMapMem);
  writer.addScalars("rho", *lbgk->getRho());
  writer.addVector("v", *lbgk->getVelocity());

  timer.start();
  for (unsigned int i = 1; i <= steps.v(); ++i) {
    lbgk->execute();
    executeAll(bc);
    if (!(i % every.v())) {
      executeAll(bcVis);
      writer.write();
    }
  }
  timer.stop();
  std::cout << "writes " << writer.getNumOfWrites() << "\n";
  std::cout << "Real Time = " << timer.realTime() << "; Processor Time = " << timer.processorTime()
            << "; Processor Load = " << timer.processorLoad() * 100 << "%" << std::endl;
  return 0;
}
