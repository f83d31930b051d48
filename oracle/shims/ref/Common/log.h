/* Stand-in for the reference log (not used on the fitness path). */
#pragma once
