// Empty stand-in for the CUDA runtime header, used only when the reference's
// device code is compiled as host C++ by oracle/build_ref.sh.
#pragma once
