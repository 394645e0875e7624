/*
 * aslb_asl_bc.hpp -- ASL's LBGK boundary conditions and surface force/flux
 * (src/num/aslLBGKBC.h:43-336 of the reference) over the C ABI. Included by
 * aslb_asl.hpp.
 *
 * A condition builds its link list in init() (initAll) from the map as it
 * stands then, and execute() launches it on the domain's stream, like ASL's
 * BCond objects (src/num/aslLBGKBC.cxx:80-83, 257-260). Conditions are
 * executed in the user's order; later writers win on shared ghost slots.
 */
#ifndef ASLB_ASL_BC_HPP
#define ASLB_ASL_BC_HPP

namespace asl {

// A condition of the library bound to one domain.
class BCLBGKCommon : public BCond {
 protected:
  SPLBGK num;
  aslb_bc* h_ = nullptr;
  virtual void create() = 0;

 public:
  explicit BCLBGKCommon(SPLBGK nm) : num(nm) {}
  ~BCLBGKCommon() override {
    if (h_) aslb_bc_destroy(h_);
  }
  void init() override {
    if (!h_) create();
  }
  void execute() override {
    init();
    aslb_detail::check(aslb_bc_execute(h_), "BCond::execute");
  }
  // extension: the library's condition handle
  aslb_bc* handle() {
    init();
    return h_;
  }
  // extension: fold a no-slip condition into the stream-collide kernel
  // (bounce-back inline; results unchanged; it must come last in its list)
  void fuse() { aslb_detail::check(aslb_bc_fuse(handle()), "BCNoSlip::fuse"); }
};

// Conditions on the walls of the block: point lists of addSliceX0 .. addSliceZE
// (src/num/aslBCond.cxx:373-510).
class BCSlices : public BCLBGKCommon {
 protected:
  unsigned mask_ = 0;
  int kind_;
  double p_ = 0.0;
  double u_[3] = {0, 0, 0};
  void create() override {
    if (!mask_) errorMessage("BCond::init: no slices were added");
    aslb_detail::check(aslb_bc_slice_create(num->handle(), kind_, mask_, p_, u_, &h_), "BCond::init");
  }

 public:
  BCSlices(SPLBGK nm, int kind) : BCLBGKCommon(nm), kind_(kind) {}
  void addSlice(SlicesNames s) {
    if (h_) errorMessage("BCond::addSlice: the condition is initialised already");
    mask_ |= ASLB_WALL((unsigned)s);
  }
  void addSliceX0() { addSlice(X0); }
  void addSliceXE() { addSlice(XE); }
  void addSliceY0() { addSlice(Y0); }
  void addSliceYE() { addSlice(YE); }
  void addSliceZ0() { addSlice(Z0); }
  void addSliceZE() { addSlice(ZE); }
  void addSlices(const std::vector<SlicesNames>& sl) {
    for (SlicesNames s : sl) addSlice(s);
  }
};

// The free forms of src/num/aslBCond.h:311-319 (programs call them on the
// condition object, e.g. addSliceX0(bcIn)).
inline void addSliceX0(BCSlices& b) { b.addSliceX0(); }
inline void addSliceXE(BCSlices& b) { b.addSliceXE(); }
inline void addSliceY0(BCSlices& b) { b.addSliceY0(); }
inline void addSliceYE(BCSlices& b) { b.addSliceYE(); }
inline void addSliceZ0(BCSlices& b) { b.addSliceZ0(); }
inline void addSliceZE(BCSlices& b) { b.addSliceZE(); }
inline void addSlices(BCSlices& b, const std::vector<SlicesNames>& sl) { b.addSlices(sl); }

// f_k(p) = f_inv(k)(q)
class BCNoSlip : public BCSlices {
 public:
  explicit BCNoSlip(SPLBGK nm) : BCSlices(nm, ASLB_BC_NOSLIP) {}
};
// f_k(p) = P
class BCConstantPressure : public BCSlices {
 public:
  acl::VectorOfElements pressure;
  BCConstantPressure(SPLBGK nm, const acl::VectorOfElements& p) : BCSlices(nm, ASLB_BC_PRESSURE), pressure(p) {
    p_ = p.value();
  }
};
// f_k(p) = f_inv(k)(q) + 6 c_k.u
class BCConstantVelocity : public BCSlices {
 public:
  acl::VectorOfElements velocity;
  BCConstantVelocity(SPLBGK nm, const acl::VectorOfElements& v) : BCSlices(nm, ASLB_BC_VELOCITY), velocity(v) {
    for (int a = 0; a < 3; ++a) u_[a] = v.value(a);
  }
};
// f_k(p) = P + 3 c_k.u
class BCConstantPressureVelocity : public BCSlices {
 public:
  acl::VectorOfElements pressure;
  acl::VectorOfElements velocity;
  BCConstantPressureVelocity(SPLBGK nm, const acl::VectorOfElements& p, const acl::VectorOfElements& v)
      : BCSlices(nm, ASLB_BC_PRESSURE_VELOCITY), pressure(p), velocity(v) {
    p_ = p.value();
    for (int a = 0; a < 3; ++a) u_[a] = v.value(a);
  }
};

// Conditions on a map (cells with -0.9999 < map <= 0 next to fluid,
// src/num/aslLBGKBC.cxx:205-438).
class BCMap : public BCLBGKCommon {
 protected:
  SPAbstractDataWithGhostNodes map_, cd_;
  int kind_;
  double p_ = 0.0;
  double u_[3] = {0, 0, 0}, om_[3] = {0, 0, 0}, c_[3] = {0, 0, 0};
  void create() override {
    const std::vector<float> m = map_->floats();
    if (cd_) {
      const std::vector<float> cd = cd_->floats();
      aslb_detail::check(aslb_bc_map_create_cd(num->handle(), kind_, m.data(), cd.data(), p_, u_, om_, c_, &h_),
                         "BCondWithMap::init");
    } else {
      aslb_detail::check(aslb_bc_map_create(num->handle(), kind_, m.data(), p_, u_, om_, c_, &h_),
                         "BCondWithMap::init");
    }
  }
  void set_velocity(const SPPositionFunction& v) {
    if (v->rotation) {
      kind_ = kind_ == ASLB_BC_MAP_VELOCITY ? ASLB_BC_MAP_VELOCITY_ROTATION : kind_;
      for (int a = 0; a < 3; ++a) {
        om_[a] = v->omega[a];
        c_[a] = v->center[a];
      }
    } else {
      for (int a = 0; a < 3; ++a) u_[a] = v->value[a];
    }
  }

 public:
  BCMap(SPLBGK nm, int kind, SPAbstractDataWithGhostNodes map) : BCLBGKCommon(nm), map_(map), kind_(kind) {}
};

class BCNoSlipMap : public BCMap {
 public:
  BCNoSlipMap(SPLBGK nm, SPAbstractDataWithGhostNodes map) : BCMap(nm, ASLB_BC_MAP_NOSLIP, map) {}
};
class BCVelocityMap : public BCMap {
 public:
  BCVelocityMap(SPLBGK nm, SPPositionFunction v, SPAbstractDataWithGhostNodes map)
      : BCMap(nm, ASLB_BC_MAP_VELOCITY, map) {
    set_velocity(v);
  }
  BCVelocityMap(SPLBGK nm, SPPositionFunction v, SPAbstractDataWithGhostNodes map,
                SPAbstractDataWithGhostNodes computationalDomain)
      : BCMap(nm, ASLB_BC_MAP_VELOCITY, map) {
    cd_ = computationalDomain;
    set_velocity(v);
  }
};
class BCConstantPressureVelocityMap : public BCMap {
 public:
  BCConstantPressureVelocityMap(SPLBGK nm, double p, const AVec<>& v, SPAbstractDataWithGhostNodes map)
      : BCMap(nm, ASLB_BC_MAP_PRESSURE_VELOCITY, map) {
    p_ = p;
    for (int a = 0; a < 3; ++a) u_[a] = v[a];
  }
};

// Conditions on the density / velocity outputs near a map, for visualisation
// (src/num/aslLBGKBC.cxx:808-852).
class BCFieldMap : public BCMap {
 protected:
  void create() override {
    const std::vector<float> m = map_->floats();
    aslb_detail::check(aslb_bc_field_create(num->handle(), kind_, m.data(), u_, om_, c_, &h_), "BCondWithMap::init");
  }

 public:
  BCFieldMap(SPLBGK nm, int kind, SPAbstractDataWithGhostNodes map) : BCMap(nm, kind, map) {}
  void velocity(const SPPositionFunction& v) {
    if (v->rotation) {
      kind_ = ASLB_BC_FIELD_VELOCITY_VEL_ROTATION;
      for (int a = 0; a < 3; ++a) {
        om_[a] = v->omega[a];
        c_[a] = v->center[a];
      }
    } else {
      for (int a = 0; a < 3; ++a) u_[a] = v->value[a];
    }
  }
};

// Deposition on a map surface (src/num/aslLBGKBC.cxx:440-598, 878-903).
class BCDepositionMap : public BCLBGKCommon {
  SPAbstractDataWithGhostNodes map_;
  int kind_;
  double p0_, lf_, beta_;
  void create() override {
    const std::vector<float> m = map_->floats();
    aslb_detail::check(aslb_bc_deposition_create(num->handle(), kind_, m.data(), p0_, lf_, beta_, &h_),
                       "BCondWithMap::init");
  }

 public:
  BCDepositionMap(SPLBGK nm, int kind, SPAbstractDataWithGhostNodes map, double p0, double lf, double beta)
      : BCLBGKCommon(nm), map_(map), kind_(kind), p0_(p0), lf_(lf), beta_(beta) {}
};

// ComputeSurfaceForceMap (src/num/aslLBGKBC.cxx:674-742): the per-cell force
// field into forceField (3 components); the FP64 totals the reference lacks
// are kept (extension: getForce / getTorque).
class ComputeSurfaceForceMap : public NumMethod {
  SPLBGK num;
  SPDataWithGhostNodesACLData forceField;
  SPAbstractDataWithGhostNodes map_;
  aslb_force* h_ = nullptr;
  double out_[6] = {0, 0, 0, 0, 0, 0};
  AVec<> r0_ = AVec<>(3, 0.);

 public:
  ComputeSurfaceForceMap(SPLBGK nm, SPDataWithGhostNodesACLData fF, SPAbstractDataWithGhostNodes map)
      : num(nm), forceField(fF), map_(map) {}
  ~ComputeSurfaceForceMap() override {
    if (h_) aslb_force_destroy(h_);
  }
  void init() override {
    if (h_) return;
    if (forceField && forceField->getEContainerSize() != 3) errorMessage("ComputeSurfaceForceMap: needs 3 components");
    const std::vector<float> m = map_->floats();
    aslb_detail::check(aslb_force_create(num->handle(), m.data(), &h_), "ComputeSurfaceForceMap::init");
  }
  void execute() override {
    init();
    const double r0[3] = {r0_[0], r0_[1], r0_[2]};
    std::vector<float> field;
    if (forceField) field.resize(3 * forceField->cells());
    aslb_detail::check(aslb_force_compute(h_, r0, forceField ? field.data() : nullptr, out_),
                       "ComputeSurfaceForceMap::execute");
    if (forceField) {
      std::vector<double>& v = forceField->values();
      for (size_t i = 0; i < field.size(); ++i) v[i] = field[i];
    }
  }
  // extension: FP64 total force and torque about r0 of the last execute()
  void setTorqueCenter(const AVec<>& r0) { r0_ = r0; }
  AVec<> getForce() const { return makeAVec(out_[0], out_[1], out_[2]); }
  AVec<> getTorque() const { return makeAVec(out_[3], out_[4], out_[5]); }
};
typedef std::shared_ptr<ComputeSurfaceForceMap> SPComputeSurfaceForceMap;

// ComputeSurfaceFluxMap (src/num/aslLBGKBC.cxx:623-665): the flux field into
// fluxField (1 component); extension: getTotal.
class ComputeSurfaceFluxMap : public NumMethod {
  SPLBGK num;
  SPDataWithGhostNodesACLData fluxField;
  SPAbstractDataWithGhostNodes map_;
  aslb_flux* h_ = nullptr;
  double total_ = 0.0;

 public:
  ComputeSurfaceFluxMap(SPLBGK nm, SPDataWithGhostNodesACLData fF, SPAbstractDataWithGhostNodes map)
      : num(nm), fluxField(fF), map_(map) {}
  ~ComputeSurfaceFluxMap() override {
    if (h_) aslb_flux_destroy(h_);
  }
  void init() override {
    if (h_) return;
    const std::vector<float> m = map_->floats();
    aslb_detail::check(aslb_flux_create(num->handle(), m.data(), &h_), "ComputeSurfaceFluxMap::init");
  }
  void execute() override {
    init();
    std::vector<float> field;
    if (fluxField) field.resize(fluxField->cells());
    aslb_detail::check(aslb_flux_compute(h_, fluxField ? field.data() : nullptr, &total_),
                       "ComputeSurfaceFluxMap::execute");
    if (fluxField) {
      std::vector<double>& v = fluxField->values();
      for (size_t i = 0; i < field.size(); ++i) v[i] = field[i];
    }
  }
  double getTotal() const { return total_; }
};

// ---- generators (src/num/aslLBGKBC.h:281-336) -------------------------------

inline SPBCond generateBCNoSlip(SPLBGK nm, const std::vector<SlicesNames>& sl) {
  auto bc = std::make_shared<BCNoSlip>(nm);
  bc->addSlices(sl);
  return bc;
}
inline SPBCond generateBCConstantVelocity(SPLBGK nm, AVec<> v, const std::vector<SlicesNames>& sl) {
  auto bc = std::make_shared<BCConstantVelocity>(nm, acl::generateVEConstant(v));
  bc->addSlices(sl);
  return bc;
}
inline SPBCond generateBCConstantPressure(SPLBGK nm, double p, const std::vector<SlicesNames>& sl) {
  auto bc = std::make_shared<BCConstantPressure>(nm, acl::generateVEConstant(p));
  bc->addSlices(sl);
  return bc;
}
inline SPBCond generateBCConstantPressureVelocity(SPLBGK nm, double p, AVec<> v, const std::vector<SlicesNames>& sl) {
  auto bc = std::make_shared<BCConstantPressureVelocity>(nm, acl::generateVEConstant(p), acl::generateVEConstant(v));
  bc->addSlices(sl);
  return bc;
}
inline SPNumMethod generateBCConstantPressure(SPLBGK nm, double p, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCConstantPressureVelocityMap>(nm, p, AVec<>(3, 0.), map);
}
inline SPNumMethod generateBCConstantPressureVelocity(SPLBGK nm, double p, AVec<> v, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCConstantPressureVelocityMap>(nm, p, v, map);
}
inline SPNumMethod generateBCNoSlip(SPLBGK nm, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCNoSlipMap>(nm, map);
}
template <class D, class = typename std::enable_if<std::is_base_of<AbstractDataWithGhostNodes, D>::value>::type>
inline SPNumMethod generateBCNoSlip(SPLBGK nm, std::shared_ptr<D> map) {
  return generateBCNoSlip(nm, std::static_pointer_cast<AbstractDataWithGhostNodes>(map));
}
inline SPNumMethod generateBCNoSlipVel(SPLBGK nm, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCFieldMap>(nm, ASLB_BC_FIELD_NOSLIP_VEL, map);
}
inline SPNumMethod generateBCNoSlipRho(SPLBGK nm, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCFieldMap>(nm, ASLB_BC_FIELD_NOSLIP_RHO, map);
}
inline SPNumMethod generateBCVelocity(SPLBGK nm, SPPositionFunction v, SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCVelocityMap>(nm, v, map);
}
inline SPNumMethod generateBCVelocity(SPLBGK nm, SPPositionFunction v, SPAbstractDataWithGhostNodes map,
                                      SPAbstractDataWithGhostNodes computationalDomain) {
  return std::make_shared<BCVelocityMap>(nm, v, map, computationalDomain);
}
inline SPNumMethod generateBCVelocityVel(SPLBGK nm, SPPositionFunction v, SPAbstractDataWithGhostNodes map) {
  auto bc = std::make_shared<BCFieldMap>(nm, ASLB_BC_FIELD_VELOCITY_VEL, map);
  bc->velocity(v);
  return bc;
}
// the argument order of the definitions (src/num/aslLBGKBC.cxx:878-903)
inline SPNumMethod generateBCTransportLimitedDeposition(SPLBGK nm, double p0, double limitingFactor,
                                                        SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCDepositionMap>(nm, ASLB_BC_MAP_TRANSPORT_DEPOSITION, map, p0, limitingFactor, 0.0);
}
inline SPNumMethod generateBCKineticsLimitedDeposition(SPLBGK nm, double p0, double limitingFactor, double beta,
                                                       SPAbstractDataWithGhostNodes map) {
  return std::make_shared<BCDepositionMap>(nm, ASLB_BC_MAP_KINETICS_DEPOSITION, map, p0, limitingFactor, beta);
}
inline SPNumMethod generateComputeSurfaceFlux(SPLBGK nm, SPDataWithGhostNodesACLData fF,
                                              SPAbstractDataWithGhostNodes map) {
  return std::make_shared<ComputeSurfaceFluxMap>(nm, fF, map);
}
inline SPNumMethod generateComputeSurfaceForce(SPLBGK nm, SPDataWithGhostNodesACLData fF,
                                               SPAbstractDataWithGhostNodes map) {
  return std::make_shared<ComputeSurfaceForceMap>(nm, fF, map);
}

}  // namespace asl

#endif  // ASLB_ASL_BC_HPP
