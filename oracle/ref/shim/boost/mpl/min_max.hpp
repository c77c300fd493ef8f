/* included by the reference's RenderingKernels.cu without use */
#pragma once
