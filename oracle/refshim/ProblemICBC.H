// Test infrastructure: stand-in for the case directory's ProblemICBC.H, which include/Tagging.H includes.
// The oracle defines no spatio-temporal tagging function, so Tagging.H uses its own empty default.
#pragma once
