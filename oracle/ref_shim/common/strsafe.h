/* Stand-in for the Windows strsafe header the reference includes
 * (CT_Recon/hf_siddon_recon.hpp:11); none of its functions are used.
 * Checker shim. */
#pragma once
