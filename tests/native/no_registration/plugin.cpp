// Test library without a problem registration.
extern "C" __attribute__((visibility("default"))) int not_a_problem() { return 0; }
