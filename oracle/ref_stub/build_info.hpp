// Stub configuration header used only when the reference is compiled as a
// test oracle (CPU, OpenMP, local-kron mode: KRON_MODE_GLOBAL left undefined).
#pragma once
#define GIT_BRANCH "oracle"
#define GIT_COMMIT_HASH "oracle"
#define GIT_COMMIT_SUMMARY "oracle"
#define BUILD_TIME "oracle"
#define ASGARD_USE_OPENMP
#define ASGARD_ENABLE_FLOAT
#define ASGARD_ENABLE_DOUBLE
#define ASGARD_SCRIPTS_DIR "./"
#define ASGARD_GOLD_BASE_DIR "./"
#define ASGARD_NUM_GPU_BLOCKS 300
#define ASGARD_NUM_GPU_THREADS 1024
#define ASGARD_NUM_QUADRATURE 10
