// Test infrastructure only.  Force-included (g++ -include) into every MPulse
// translation unit of the oracle build, together with
// -DMPULSE_FOCUSEDPULSEINJECT_H, which makes the real focusedpulseinject.h a
// no-op.  That header and focusedpulseinject.cpp / focusedpulsefunctions.cpp do
// not compile upstream (duplicate members at focusedpulseinject.h:116-132,
// undeclared names at focusedpulsefunctions.cpp:49-145, FocusedPulseDataGenerator::
// init declared at focusedpulseinject.h:83 and never defined).  fdtd_plrc.t:459-461
// still registers "focused_pulse_inject", so a class of that name must exist; this
// one refuses to run, exactly like a setup file naming a broken plug-in should.
#ifndef MPB_REFSHIM_FOCUSED_STUB_H
#define MPB_REFSHIM_FOCUSED_STUB_H
#ifdef __cplusplus
#include <cstdlib>
#include <iostream>
#include "currentfactory.h"

class FocusedPulseInject : public CurrentFactory {
 public:
  virtual ~FocusedPulseInject() {}
  void initCurrents(Storage *, FieldSolver *) {
    std::cerr << "focused_pulse_inject: not available, the upstream source does not compile\n";
    std::exit(-1);
  }
};
#endif
#endif
