// batch.cuh — batched ensemble of independent scenes (see batch.cu).
#pragma once
#include "simulator.cuh"
