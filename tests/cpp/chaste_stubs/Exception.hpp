#pragma once
#include "chaste_stub_core.hpp"
