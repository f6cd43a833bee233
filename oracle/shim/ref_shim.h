/*
 * Force-included header for compiling the reference's own FD sources
 * (src/util/{fd,InitInversion,global,wavelet}.cpp) with g++ 13 as a CPU
 * oracle.  Test infrastructure only: nothing in the shipped library links it.
 *
 * Why it exists:
 *  - src/util/debug.h:19,27,28 does not compile under a modern g++ (an
 *    unqualified `cout` inside a template, an undeclared `i3`).  Defining its
 *    include guard DEBUG_H_H here skips that header; the declarations below
 *    replace it with the same names and signatures (debug.h:5-6).
 *  - src/util/debug.cpp:5-12 calls exit(0) on a failed check, which would end a
 *    test process silently.  ref_shim.cpp defines check()/error() so that a
 *    failed check throws instead; the call sites are unchanged.
 */
#ifndef SEIS_REF_SHIM_H
#define SEIS_REF_SHIM_H
#include <iostream>
#include <string>
#include <cstdio>
#define DEBUG_H_H 1
using std::cout;
using std::endl;
void check(bool eval, char *str);
void error(std::string errinfo);
#endif
