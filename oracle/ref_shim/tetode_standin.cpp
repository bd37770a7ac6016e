// Project-written stand-in for the reference's deterministic solver TetODE
// (src/steps/tetode/tetode.cpp), which needs the SUNDIALS CVODE library, absent here.  The
// reference's Python binding (pysteps/cysteps_solver.pyx, class
// _py_TetODE) calls three of its members; here they throw instead of building the
// solver, so the binding module loads and every other class in it works.  The symbols are
// the members' own (Itanium-mangled) names; all arguments are pointers, integers or
// doubles, passed as the members receive them.
#include <stdexcept>

namespace {
[[noreturn]] void tetode_absent() {
    throw std::runtime_error("TetODE needs the SUNDIALS CVODE library, which is absent");
}
}  // namespace

// steps::tetode::TetODE::TetODE(model::Model*, wm::Geom*, const rng::RNGptr&, int)
void tetode_ctor(void*, void*, void*, const void*, int) __asm__(
    "_ZN5steps6tetode6TetODEC1EPNS_5model5ModelEPNS_2wm4GeomERKSt10shared_ptrINS_3rng3RNGEEi");
void tetode_ctor(void*, void*, void*, const void*, int) {
    tetode_absent();
}
// steps::tetode::TetODE::setTolerances(double, double)
void tetode_set_tolerances(void*, double, double) __asm__("_ZN5steps6tetode6TetODE13setTolerancesEdd");
void tetode_set_tolerances(void*, double, double) {
    tetode_absent();
}
// steps::tetode::TetODE::setMaxNumSteps(unsigned int)
void tetode_set_max_num_steps(void*, unsigned int) __asm__("_ZN5steps6tetode6TetODE14setMaxNumStepsEj");
void tetode_set_max_num_steps(void*, unsigned int) {
    tetode_absent();
}
