/* Fermion-parity function for the bosonic oracle builds.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference applies fermionic signs from the
 * legs' directions whether or not the model is fermionic (src/qtensor.cpp:816,
 * :953, :962, :1084); the directions are stamped by svd() on every model
 * (src/qtensor.cpp:1149-1151).  For the bosonic models (XYZ, Potts) that makes
 * H_eff non-Hermitian.  Those sign sites all have the form
 * 1-2*((ff(x)*ff(y))%2), so building the bosonic variants with the parity
 * function ff (src/useful.cpp:32) replaced by zero gives sign = +1 at every
 * site: exactly the reference with its sign code compiled out, and nothing else
 * changed.  The reference's own ff is renamed at compile time for these builds.
 */
int ff(int) { return 0; }
