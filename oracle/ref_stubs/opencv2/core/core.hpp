/* Stand-in: the reference headers on the solver path only name cv::Mat in declarations. */
#pragma once
namespace cv { class Mat; }
