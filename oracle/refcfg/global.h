/* Build configuration for compiling the reference DMRG sources as the oracle.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the product links against this.
 *
 * The reference takes its compile-time switches from a `global.h` at its root
 * (clover199/DMRG global.h:14-25).  This header stands in for it so that the
 * reference sources can be built unmodified, where they lie, for each symmetry
 * configuration.  The switches come from the compiler command line:
 *   -DORACLE_SYMMETRY=<N>   Z_N fusion rule (2 Kitaev/XYZ, 3 Potts, 32 U(1) embedding)
 *   -DORACLE_FERMION        fermionic operators and signs (Kitaev, S4E)
 *   -DORACLE_S4E            Z2 x Z2 x Z2 fusion rule and parity table (with SYMMETRY 8)
 *   -DORACLE_PBC            periodic boundary: edge environments (global.h:14 PBC)
 * The numerical constants (TOL, NEV, ...) keep the values the reference ships
 * with, because the reference's ARPACK wrapper and printers read them.
 */
#ifndef _MY_GLOBAL_
#define _MY_GLOBAL_

#include <iostream>
#include <fstream>
#include <sstream>
#include <complex>
#include <vector>
#include <string>
#include <cmath>
#include <cstdlib>
#include <ctime>

#ifndef ORACLE_SYMMETRY
#error "ORACLE_SYMMETRY must be given on the command line"
#endif
#define SYMMETRY ORACLE_SYMMETRY
#ifdef ORACLE_FERMION
#define FERMION
#endif
#ifdef ORACLE_S4E
#define S4E
#endif
#ifdef ORACLE_PBC
#define PBC
#endif

#define TOL 1e-10
#define ACC 10
#define NEV 6
#define NSI 20
#define ZERO 0.01
#define PRINT_TO_SCREEN 0
#define PI 3.14159265359

using std::cout;
using std::endl;
using std::cerr;
using std::ofstream;
using std::ifstream;
using std::fstream;
using std::ios;
using std::vector;
using std::complex;
using std::string;
using std::abs;

#endif
