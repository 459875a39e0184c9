/*
 * Override of the reference's include/ComputeConfig.hpp for the CPU oracle
 * build: the reference's own CPU path (use_cuda=false) with load balancing off,
 * exactly the branch src/Euler.cpp:462-493 takes when no GPU is used.
 */
#pragma once
inline constexpr bool use_cuda = false;
inline constexpr bool enable_dlb = false;
