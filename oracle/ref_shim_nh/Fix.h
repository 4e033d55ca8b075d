// Test infrastructure only (oracle/ref_nh_harness.cu, oracle/ref_berendsen_harness.cu).
// Stand-in for the reference's Fix.h: the base-class members the barostats use
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <boost/python.hpp>
#include <boost/shared_ptr.hpp>
#include "Bond.h"
#include "Virial.h"
class State;
class Fix {
public:
    State *state;
    std::string handle, groupHandle, type;
    uint32_t groupTag = 1;
    bool prepared = false;
    bool requiresPostNVE_V = false, requiresForces = false, isThermostat = false, requiresVirials = false,
         requiresPerAtomVirials = false;
    int virialMode = 0;
    template <class... A>
    Fix(boost::shared_ptr<State> s, std::string h, std::string g, std::string t, A...)
        : state(s.get()), handle(h), groupHandle(g), type(t) {}
    virtual ~Fix() {}
    virtual void updateScaleVariables() {}
    virtual std::vector<BondVariant> *getBonds() { return nullptr; }
};
