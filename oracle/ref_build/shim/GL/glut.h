// Intentionally empty: no windowing or GL entry points are provided.
#pragma once
