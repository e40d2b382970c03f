// See dccrg.hpp in this folder.
#pragma once
#include "dccrg.hpp"
