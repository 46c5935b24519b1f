/* Stand-in for the CUDA-samples timer header the reference includes
 * (CT_Recon/hf_siddon_class.hpp:13).  Nothing from it is used by the code
 * compiled here (only mlem.cu uses StopWatchInterface).  Checker shim. */
#pragma once
