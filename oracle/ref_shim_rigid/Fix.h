// Test infrastructure only (oracle/ref_rigid_harness.cu).
// Stand-in for the reference's Fix.h: the base-class members FixRigid.cu uses
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <pugixml.hpp>
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
    bool requiresPostNVE_V = false, requiresForces = false;
    int virialMode = 0;
    Fix(boost::shared_ptr<State> s, std::string h, std::string g, std::string t, bool, bool, bool, int)
        : state(s.get()), handle(h), groupHandle(g), type(t) {}
    virtual ~Fix() {}
    pugi::xml_node getRestartNode() { return pugi::xml_node(); }
    virtual std::vector<BondVariant> *getBonds() { return nullptr; }
};
