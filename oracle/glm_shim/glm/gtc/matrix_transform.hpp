// ORACLE -- test infrastructure only. Empty: the reference headers include
// this GLM header but the BVH build uses nothing from it.
#pragma once
#include "../glm.hpp"
