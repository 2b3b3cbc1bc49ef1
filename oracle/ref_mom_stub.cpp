// Stand-in for the reference's GPU table upload, so that its driver (mom.cpp)
// runs on the CPU path: mom.cpp:187 calls setup_gpu() unconditionally.  Test
// infrastructure only.
void setup_gpu() {}
