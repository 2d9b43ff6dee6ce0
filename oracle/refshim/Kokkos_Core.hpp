// Empty stand-in: lets the reference header master_element/Hex8GeometryFunctions.h
// compile without Kokkos/STK for the oracle/_ref geometry check.
#pragma once
