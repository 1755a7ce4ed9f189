// Empty stand-in: the reference kernels include rapidjson through
// parameters_sim.h but use none of it (TEST INFRASTRUCTURE).
#pragma once
