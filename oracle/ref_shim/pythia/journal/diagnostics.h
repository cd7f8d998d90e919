/* Shim: the journal macros are referenced by headers but never expanded in
 * the pointwise kernels the oracle calls. Test infrastructure only. */
#pragma once
#define __HERE__ __FILE__, __LINE__, __func__
