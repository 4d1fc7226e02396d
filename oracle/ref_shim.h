/* Forced-include shim for compiling the reference's host arithmetic
 * (include/host-arith/**, src/host-arith/**) with plain g++ instead of nvcc.
 * The reference relies on headers that nvcc pulls in implicitly; nothing
 * else changes.  Test infrastructure only: used by oracle/Makefile to build
 * oracle/_ref/libref.so, the reference's own CPU arithmetic. */
#pragma once
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <algorithm>
#include <vector>
using std::max;
