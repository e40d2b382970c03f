// Empty stand-in for the reference's grid.h (oracle builds only).
#pragma once
