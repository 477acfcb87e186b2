// Test infrastructure only (oracle). Empty stand-in for the C++Builder VCL
// umbrella header so that the reference's TlmSolver.cpp and Geometry.cpp
// compile headless with g++. Neither file uses a VCL symbol on the TLM path.
#pragma once
