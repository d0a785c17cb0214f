/* Drop-in path of qkrylov's C ABI header: the declarations live in
 * qkrylov_c_api.h at the top of the include directory. */
#include "../qkrylov_c_api.h"
