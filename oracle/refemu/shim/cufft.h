// Empty stand-in so the reference kernels compile as host C++ (oracle test infrastructure).
#pragma once
