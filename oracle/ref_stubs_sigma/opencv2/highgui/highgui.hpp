/* Stand-in: included by the reference's depth-noise model, which uses none of it. */
#pragma once
