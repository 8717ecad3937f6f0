#pragma once
// Drop-in for the reference's include/Trajectory.hpp:7: one extended-XYZ frame in stable-id order.

#include "System.hpp"

#include <cstdio>

void writeXyzFrame(std::FILE* file, const System& system, double time);
