// Test infrastructure only (oracle/ref_ewald_harness.cu).
// Stand-in for the reference's Fix.h: the base-class members FixCharge,
// FixChargeEwald and the evaluator wrappers they build use
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <boost/python.hpp>
#include <boost/shared_ptr.hpp>
#include "Bond.h"
#include "Virial.h"
class State;
class EvaluatorWrapper;
class Fix {
public:
    State *state;
    std::string handle, groupHandle, type;
    uint32_t groupTag = 1;
    bool prepared = false, forceSingle = false, requiresCharges = false;
    bool canOffloadChargePairCalc = false, hasOffloadedChargePairCalc = false;
    bool requiresVirials = false, requiresPerAtomVirials = false;
    std::string evalWrapperMode = "self";
    boost::shared_ptr<EvaluatorWrapper> evalWrap;
    int nThreadPerBlock() { return 256; }
    int nThreadPerAtom() { return 1; }
    int applyEvery = 1, orderPreference = 0;
    template <class... A>
    Fix(boost::shared_ptr<State> s, std::string h, std::string g, std::string t, A...)
        : state(s.get()), handle(h), groupHandle(g), type(t) {}
    virtual ~Fix() {}
    virtual bool handleLocalData() { return true; }
    virtual std::vector<BondVariant> *getBonds() { return nullptr; }
    virtual void compute(int) {}
    virtual void singlePointEng(real *) {}
    virtual void singlePointEngGroupGroup(real *, uint32_t, uint32_t) {}
    virtual void setEvalWrapper() {}
    virtual bool prepareForRun() { return true; }
    virtual std::vector<real> getRCuts() { return {}; }
    virtual void handleBoundsChange() {}
};
