// Minimal stand-in for waLBerla's core/Macros.h: only the restrict qualifier.  Test infrastructure only.
#pragma once
#define WALBERLA_RESTRICT __restrict__
