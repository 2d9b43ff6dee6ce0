// Oracle (test infrastructure only): empty stand-in for the reference's
// src/controls/controls.h (nothing of it is used by assembler.h's code paths
// compiled here).
#pragma once
