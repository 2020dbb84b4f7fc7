// Stand-in for the CUDA-samples helper header the reference includes (unused).
#pragma once
