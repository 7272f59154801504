// Empty stand-in for optix_stubs.h (host build of the reference's shading headers).
#pragma once
