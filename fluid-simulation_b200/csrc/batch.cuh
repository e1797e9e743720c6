// batch.cuh — batched ensemble of independent scenes (batch.cu).
#pragma once
#include "simulator.cuh"
